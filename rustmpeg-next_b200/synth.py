"""Seeded synthetic workloads for the frame path.

- ``value_noise_frame``: the 1920x1080 10-bit 4:2:0 content of the full-frame
  configuration (4-octave value noise with octave gains 1, .5, .25, .125,
  amplitude 0..1023, translated by (+1.25, -0.75) px per frame, plus 8 moving
  64x64 textured rectangles with velocities uniform in +-6 px/frame; chroma is
  the same noise at half resolution scaled to [384, 640]).
- ``random_records``: decoder inputs with the statistics of coded pictures
  (per-CU intra modes, CCLM chroma modes, sparse low-frequency transform levels
  whose density falls with frequency and QP, per-CTU SAO parameters and ALF
  switches), for picture batches of any size, bit depth and chroma format.

Seeds follow 0x5EED0000 + stream * 1000 + frame.
"""
from __future__ import annotations

import numpy as np

from . import (APS_DTYPE, CTU_DTYPE, CU_DTYPE, PIC_DTYPE, TOOL_ALF, TOOL_DEBLOCK, TOOL_DEP_QUANT,
               TOOL_ENC_CCLM, TOOL_ENC_FULL_INTRA, TOOL_SAO, TOOL_SPARSE_LEVELS, TOOL_TU_TOOLS, chroma_dims)


def seed_for(stream: int, frame: int) -> int:
    return 0x5EED0000 + stream * 1000 + frame


def _value_noise(h, w, cell, rng_seed, ox=0.0, oy=0.0):
    rng = np.random.default_rng(rng_seed)
    gh, gw = int((h + abs(oy)) / cell) + 3, int((w + abs(ox)) / cell) + 3
    lattice = rng.random((gh, gw))
    ys = (np.arange(h)[:, None] + oy) / cell + 1
    xs = (np.arange(w)[None, :] + ox) / cell + 1
    y0 = np.floor(ys).astype(int)
    x0 = np.floor(xs).astype(int)
    fy = ys - y0
    fx = xs - x0
    fy = fy * fy * (3 - 2 * fy)
    fx = fx * fx * (3 - 2 * fx)
    y0 = np.clip(y0, 0, gh - 2)
    x0 = np.clip(x0, 0, gw - 2)
    a = lattice[y0, x0]
    b = lattice[y0, x0 + 1]
    c = lattice[y0 + 1, x0]
    d = lattice[y0 + 1, x0 + 1]
    return (a * (1 - fx) + b * fx) * (1 - fy) + (c * (1 - fx) + d * fx) * fy


def _noise(h, w, seed, ox, oy, base_cell=128.0):
    acc = np.zeros((h, w))
    norm = 0.0
    for o, g in enumerate((1.0, 0.5, 0.25, 0.125)):
        acc += g * _value_noise(h, w, base_cell / (2 ** o), seed + 17 * o, ox / (2 ** 0), oy)
        norm += g
    return acc / norm


def value_noise_frame(w=1920, h=1080, bd=10, frame=0, stream=0):
    """One frame of the full-frame content; returns (y, u, v) uint16 planes."""
    mx = (1 << bd) - 1
    base = seed_for(stream, 0)
    ox, oy = 1.25 * frame, -0.75 * frame
    y = _noise(h, w, base, ox, oy) * mx
    rng = np.random.default_rng(base + 7)
    pos = rng.uniform([0, 0], [w - 64, h - 64], size=(8, 2))
    vel = rng.uniform(-6, 6, size=(8, 2))
    tex = [_noise(64, 64, base + 100 + k, 0, 0, base_cell=16.0) * mx for k in range(8)]
    for k in range(8):
        px, py = pos[k] + vel[k] * frame
        px = int(round(px)) % max(1, w - 64)
        py = int(round(py)) % max(1, h - 64)
        y[py:py + 64, px:px + 64] = tex[k]
    cw, ch = (w + 1) // 2, (h + 1) // 2
    lo, hi = 384 << (bd - 10) if bd >= 10 else 384 >> (10 - bd), 640 << (bd - 10) if bd >= 10 else 640 >> (10 - bd)
    u = lo + _noise(ch, cw, base + 1, ox / 2, oy / 2) * (hi - lo)
    v = lo + _noise(ch, cw, base + 2, ox / 2, oy / 2) * (hi - lo)
    return (np.clip(np.rint(y), 0, mx).astype(np.uint16), np.clip(np.rint(u), 0, mx).astype(np.uint16),
            np.clip(np.rint(v), 0, mx).astype(np.uint16))


def config1_frame(frame, stream=0, size=64):
    """One frame of the 8-bit 4:2:0 small-picture configuration: luma a
    horizontal ramp 16 -> 235 plus integer noise U[-8, 8] and a 16x16 square
    of value 200 that moves +2 px per frame (from x = 8, y = 24); chroma
    128 + U[-4, 4]. Returns (y, u, v) uint8."""
    rng = np.random.default_rng(seed_for(stream, frame))
    x = np.arange(size)
    ramp = np.rint(16 + 219 * x / (size - 1)).astype(np.int32)
    y = ramp[None, :] + rng.integers(-8, 9, (size, size))
    x0 = 8 + 2 * frame
    y[24:40, x0:x0 + 16] = 200
    y = y.clip(0, 255).astype(np.uint8)
    u = (128 + rng.integers(-4, 5, (size // 2, size // 2))).astype(np.uint8)
    v = (128 + rng.integers(-4, 5, (size // 2, size // 2))).astype(np.uint8)
    return y, u, v


def strict_picture(width, height, qp, cu_offset=0):
    """A PIC_DTYPE record for a strict 8-bit 4:2:0 picture (slice.rs:458
    decode_picture) on the frame path: CTU 32, per-TB transform tools, no
    loop filters."""
    p = np.zeros((), PIC_DTYPE)
    p["width"], p["height"] = width, height
    p["visible_width"], p["visible_height"] = width, height
    p["bit_depth"], p["chroma_format"], p["ctu_log2"] = 8, 1, 5
    p["slice_qp"] = qp
    p["chroma_qp_scaled"] = chroma_qp_scaled(qp, 8)  # derived_chroma_qp (hls.rs:778), 8-bit
    p["tools"] = TOOL_TU_TOOLS
    p["alf_aps"] = -1
    p["cu_offset"] = cu_offset
    return p


def pad_to(plane, w, h):
    """Edge-replicate a plane to (h, w) (mod.rs:2753 pad_vvc_frame)."""
    ph, pw = plane.shape
    return np.pad(plane, ((0, h - ph), (0, w - pw)), mode="edge")


def _tb_levels(rng, n, w, h, qp_scaled):
    """n TBs of sparse levels concentrated at low frequencies; density falls
    with QP; every TB keeps at least its DC level (it is coded, cbf = 1)."""
    yy, xx = np.mgrid[0:h, 0:w]
    freq = (xx + yy) / (w + h)
    dens = np.clip(0.9 * np.exp(-freq * 9.0) * np.exp(-(qp_scaled - 22) / 14.0), 0.0, 0.95)
    scale = 1.0 + 6.0 * np.exp(-freq * 6.0) * np.exp(-(qp_scaled - 22) / 12.0)
    mask = rng.random((n, h, w), dtype=np.float32) < dens
    mag = np.floor(rng.standard_exponential((n, h, w), dtype=np.float32) * scale).astype(np.int16) + 1
    sign = np.where(rng.random((n, h, w), dtype=np.float32) < 0.5, -1, 1).astype(np.int16)
    lv = (mask * mag * sign).astype(np.int16)
    empty = ~lv.reshape(n, -1).any(axis=1)
    lv[empty, 0, 0] = 1
    return lv


def random_records(pics_spec, seed=0, tools=TOOL_DEBLOCK, sao_prob=0.6, alf_aps=False,
                   sao_class3_on_edges=False):
    """Build a batch of decoder records.

    pics_spec: iterable of dicts with keys width, height (coded, CTU multiples),
    visible_width, visible_height, bit_depth, chroma_format, ctu_log2, qp.
    SAO edge class 3 is kept off the first and last CTU rows unless
    sao_class3_on_edges (the reference aborts on it there).
    Returns (pics, cus, levels, ctus, aps).
    """
    rng = np.random.default_rng(seed)
    pics, cu_chunks, lv_chunks, ctu_chunks = [], [], [], []
    n_cu = n_lv = n_ctu = 0
    for spec in pics_spec:
        w, h, bd, cf = spec["width"], spec["height"], spec["bit_depth"], spec["chroma_format"]
        ctu_log2, qp = spec.get("ctu_log2", 5), spec["qp"]
        ctu = 1 << ctu_log2
        tb = min(ctu, 32)
        sw = 2 if cf in (1, 2) else 1
        sh = 2 if cf == 1 else 1
        tcw, tch = (max(tb // sw, 2), max(tb // sh, 2)) if cf else (0, 0)
        off = 6 * (bd - 8)
        lqp = max(min(63 + off, qp + off), 4)
        qpc = min(63, max(-off, qp))
        cqp = max(0, (qpc if qpc <= 26 else qpc - 1) + off)
        p = np.zeros((), PIC_DTYPE)
        p["width"], p["height"] = w, h
        p["visible_width"] = spec.get("visible_width", w)
        p["visible_height"] = spec.get("visible_height", h)
        p["bit_depth"], p["chroma_format"], p["ctu_log2"] = bd, cf, ctu_log2
        p["slice_qp"], p["chroma_qp_scaled"] = qp, cqp
        p["tools"] = spec.get("tools", tools)
        p["alf_aps"] = 0 if alf_aps else -1
        p["cu_offset"], p["ctu_offset"] = n_cu, n_ctu
        gw, gh = w // tb, h // tb
        cus = np.zeros(gw * gh, CU_DTYPE)
        cus["luma_mode"] = rng.integers(0, 67, gw * gh)
        chm = rng.integers(0, 70, gw * gh)
        chm = np.where(chm >= 67, 81 + (chm - 67), cus["luma_mode"])
        cus["chroma_mode"] = chm if cf else 0
        ncu = gw * gh
        lo = np.full((ncu, 3), -1, np.int32)
        cbf = np.zeros(ncu, np.uint8)
        for c in range(3 if cf else 1):
            coded = rng.random(ncu) < (0.85 if c == 0 else 0.5) * np.exp(-(qp - 22) / 30.0)
            idx = np.nonzero(coded)[0]
            bw, bh = (tb, tb) if c == 0 else (tcw, tch)
            if len(idx):
                lv = _tb_levels(rng, len(idx), bw, bh, lqp if c == 0 else cqp)
                lo[idx, c] = n_lv + np.arange(len(idx), dtype=np.int64) * (bw * bh)
                lv_chunks.append(lv.reshape(-1))
                n_lv += lv.size
            cbf |= (coded.astype(np.uint8) << c)
        cus["level_off"] = lo
        cus["cbf"] = cbf
        ctus = random_ctu_params(rng, w, h, ctu, bd, cf, sao_prob, sao_class3_on_edges)
        pics.append(p)
        cu_chunks.append(cus)
        ctu_chunks.append(ctus)
        n_cu += len(cus)
        n_ctu += len(ctus)
    aps = None
    if alf_aps:
        aps = synthetic_aps(rng)
    levels = np.concatenate(lv_chunks) if lv_chunks else np.zeros(0, np.int16)
    return (np.array(pics, PIC_DTYPE), np.concatenate(cu_chunks), levels,
            np.concatenate(ctu_chunks), aps)


def random_ctu_params(rng, w, h, ctu, bd, cf, sao_prob=0.6, sao_class3_on_edges=False, alf_prob=0.7):
    """Per-CTU SAO parameters (band offset or one of the 4 edge classes per
    component, offsets within the ranges the syntax allows at this bit depth)
    and ALF luma switches for one w x h picture, CTU_DTYPE records in raster
    order. SAO edge class 3 is kept off the first and last CTU rows unless
    sao_class3_on_edges (the reference aborts on it there)."""
    nctu = (h // ctu) * (w // ctu)
    ctus = np.zeros(nctu, CTU_DTYPE)
    omax = (1 << (min(bd, 10) - 5)) - 1
    row = np.arange(nctu) // (w // ctu)
    edge_row = (row == 0) | (row == h // ctu - 1)
    for c in range(3 if cf else 1):
        r = rng.random(nctu)
        band = r < sao_prob / 2
        edge = (r >= sao_prob / 2) & (r <= sao_prob)
        eo = rng.integers(0, 4, nctu)
        if not sao_class3_on_edges:
            eo = np.where((eo == 3) & edge_row, 2, eo)
        o = rng.integers(0, omax + 1, (nctu, 4))
        ob = rng.integers(-omax, omax + 1, (nctu, 4))
        s = ctus["sao"][:, c]
        s["type"] = np.where(band, 1, np.where(edge, 2, 0))
        s["band_or_class"] = np.where(band, rng.integers(0, 32, nctu), np.where(edge, eo, 0))
        s["offsets"] = np.where(band[:, None], ob,
                                np.where(edge[:, None], o * np.array([1, 1, -1, -1]), 0))
        ctus["sao"][:, c] = s
    ctus["alf_luma"] = rng.random(nctu) < alf_prob
    return ctus


def synthetic_aps(rng, n_filters=25, luma_clip=True):
    """An ALF APS whose luma filters are fixed-filter coefficient sets of the
    standard (clip indices uniform over 0..3)."""
    from .tables import alf_fixed_coeff

    fixed = alf_fixed_coeff()
    aps = np.zeros(1, APS_DTYPE)
    aps["num_luma_filters"] = n_filters
    aps["luma_clip"] = int(luma_clip)
    aps["coeff_delta_idx"][0] = rng.integers(0, n_filters, 25)
    aps["coeff"][0, :n_filters] = fixed[rng.integers(0, 64, n_filters), :12]
    aps["clip_idx"][0, :n_filters] = rng.integers(0, 4, (n_filters, 12))
    return aps


# Shapes (log2 w, log2 h) of the transform units a random QT/MT tiling of
# 4x4..64x64 blocks produces, with the luma/chroma weights of 4:2:0, plus the
# narrow shapes ISP and 2xN chroma give.
_TU_SHAPES = [(a, b) for a in range(2, 7) for b in range(2, 7) if abs(a - b) <= 2]
_TU_ODD_SHAPES = [(0, 4), (4, 0), (0, 3), (1, 3), (3, 1), (1, 2), (2, 1), (1, 1), (0, 1), (1, 0), (1, 4),
                  (0, 6), (6, 0), (1, 5), (5, 1)]


def random_tu_records(n, seed=0, forward=False, bit_depths=(8, 10), qp_range=(22, 37), odd_frac=0.05,
                      tools=True):
    """Seeded transform-unit records (TU_DTYPE) and their int16 inputs.

    Inverse (forward=False): sparse low-frequency levels, a few at the int16
    limits. Forward: residuals of +-2^bd range with a smooth component.
    `tools` mixes in DQ, transform skip, BDPCM, implicit / explicit MTS and
    LFNST where the unit's shape allows them. Returns (recs, data, out_count).
    """
    from . import TU_DTYPE, TU_BDPCM_HOR, TU_BDPCM_VER, TU_DEP_QUANT, TU_IMPLICIT_MTS, TU_INTER, \
        TU_TRANSFORM_SKIP

    rng = np.random.default_rng(seed)
    recs = np.zeros(n, TU_DTYPE)
    shapes = np.array(_TU_SHAPES)[rng.integers(0, len(_TU_SHAPES), n)]
    odd = rng.random(n) < odd_frac
    shapes[odd] = np.array(_TU_ODD_SHAPES)[rng.integers(0, len(_TU_ODD_SHAPES), int(odd.sum()))]
    recs["log2_w"], recs["log2_h"] = shapes[:, 0], shapes[:, 1]
    bd = np.array(bit_depths)[rng.integers(0, len(bit_depths), n)]
    recs["bit_depth"] = bd
    qp = rng.integers(qp_range[0], qp_range[1] + 1, n) + 6 * (bd - 8)
    recs["qp"] = np.clip(qp, 0, 87)
    w, h = 1 << shapes[:, 0], 1 << shapes[:, 1]
    size = w * h
    if tools:
        r = rng.random(n)
        mts_ok = (w >= 4) & (h >= 4) & (w <= 32) & (h <= 32)
        lfnst_ok = (w >= 4) & (h >= 4)
        ts_ok = (w <= 32) & (h <= 32)
        flags = np.where(rng.random(n) < 0.5, TU_DEP_QUANT, 0)
        ts = ts_ok & (r < 0.15)
        flags = np.where(ts, TU_TRANSFORM_SKIP, flags)
        if not forward:
            bd_dir = rng.integers(0, 3, n)
            flags = np.where(ts & (bd_dir == 1), flags | TU_BDPCM_HOR, flags)
            flags = np.where(ts & (bd_dir == 2), flags | TU_BDPCM_VER, flags)
        mts = mts_ok & ~ts & (r >= 0.15) & (r < 0.4)
        recs["mts_idx"] = np.where(mts, rng.integers(1, 5, n), 0)
        lf = lfnst_ok & ~ts & (r >= 0.4) & (r < 0.65)
        recs["lfnst_idx"] = np.where(lf, rng.integers(1, 3, n), 0)
        recs["lfnst_mode"] = rng.integers(0, 95, n)
        imp = ~ts & (r >= 0.65) & (r < 0.8)
        flags = np.where(imp, flags | TU_IMPLICIT_MTS, flags)
        if forward:
            flags = np.where(rng.random(n) < 0.3, flags | TU_INTER, flags)
        recs["flags"] = flags
    offs = np.zeros(n + 1, np.int64)
    offs[1:] = np.cumsum(size)
    recs["in_off"] = offs[:-1]
    recs["out_off"] = offs[:-1]
    total = int(offs[-1])
    data = np.zeros(total, np.int16)
    for i in range(n):
        ww, hh, o = int(w[i]), int(h[i]), int(offs[i])
        if forward:
            amp = 1 << int(bd[i])
            yy, xx = np.mgrid[0:hh, 0:ww]
            smooth = (amp // 4) * np.sin(xx * rng.random() + yy * rng.random() + rng.random() * 6)
            v = smooth + rng.integers(-amp // 2, amp // 2 + 1, (hh, ww))
            data[o:o + ww * hh] = np.clip(v, -amp, amp).astype(np.int16).reshape(-1)
        else:
            k = min(ww * hh, 1 + int(rng.geometric(0.15)))
            ys = np.minimum((rng.exponential(hh / 6, k)).astype(int), hh - 1)
            xs = np.minimum((rng.exponential(ww / 6, k)).astype(int), ww - 1)
            mag = rng.geometric(0.35, k) * rng.choice([-1, 1], k)
            big = rng.random(k) < 0.01
            mag = np.where(big, rng.choice([-32768, 32767], k), mag)
            blk = np.zeros((hh, ww), np.int32)
            blk[ys, xs] = mag
            data[o:o + ww * hh] = np.clip(blk, -32768, 32767).astype(np.int16).reshape(-1)
    return recs, data, total


def source_planes(w, h, bd=10, cf=1, seed=0, vis=None):
    """Coded-size (w x h) source planes of value-noise content at bit depth bd
    and chroma format cf; the visible part is vis = (vw, vh), the rest is the
    reference's edge padding."""
    vw, vh = vis or (w, h)
    y, u, v = value_noise_frame(vw, vh, 10, frame=seed)

    def scale(p):
        return (p.astype(np.int32) << bd >> 10).astype(np.uint16) if bd > 10 else (p >> (10 - bd)).astype(np.uint16)

    if bd != 10:
        y, u, v = scale(y), scale(u), scale(v)
    if cf == 0:
        return pad_to(y, w, h), None, None
    sw = 2 if cf in (1, 2) else 1
    sh = 2 if cf == 1 else 1
    cw, ch = (w + sw - 1) // sw, (h + sh - 1) // sh
    if cf == 3:
        u = np.kron(u, np.ones((2, 2), np.uint16))[:vh, :vw]
        v = np.kron(v, np.ones((2, 2), np.uint16))[:vh, :vw]
    elif cf == 2:
        u = np.repeat(u, 2, axis=0)[:vh]
        v = np.repeat(v, 2, axis=0)[:vh]
    return pad_to(y, w, h), pad_to(u, cw, ch), pad_to(v, cw, ch)


def random_lmcs_aps(rng):
    """A seeded LMCS APS (LMCS_APS_DTYPE) with codeword deltas within the
    range the syntax allows for the active bins."""
    from . import LMCS_APS_DTYPE

    a = np.zeros((), LMCS_APS_DTYPE)
    lo = int(rng.integers(0, 4))
    hi = int(rng.integers(12, 16))
    a["min_bin_idx"], a["max_bin_idx"] = lo, hi
    a["bin_cw_delta"] = rng.integers(-12, 13, 16)
    a["chroma_res_scaling_offset"] = int(rng.integers(-7, 8))
    return a


def _split_tree(rng, x, y, w, h, pic_w, pic_h, min_size, out, leaf_bias, cout=None, chroma_done=False):
    """Random QT / BT / TT coding tree over one node; nodes that cross the
    picture's right or bottom edge split implicitly (halves), leaves go to out.
    With cout, chroma stops splitting at the first node with a child narrower
    or shorter than 8 luma samples (4:2:0 chroma blocks of 4x4 or more) and
    its chroma leaves go to cout."""
    cross_x, cross_y = x + w > pic_w, y + h > pic_h
    if x >= pic_w or y >= pic_h:
        return

    def chroma_at(children_min):
        # chroma of this node stays whole when a child would be below 8 luma
        if cout is not None and not chroma_done and children_min < 8:
            cout.append((x, y, w, h))
            return True
        return chroma_done

    if cross_x or cross_y:
        if cross_x and cross_y and w > min_size and h > min_size:
            cd = chroma_at(min(w, h) // 2)
            for dy in (0, h // 2):
                for dx in (0, w // 2):
                    _split_tree(rng, x + dx, y + dy, w // 2, h // 2, pic_w, pic_h, min_size, out, leaf_bias, cout, cd)
            return
        if cross_x and w > min_size:
            cd = chroma_at(min(w // 2, h))
            _split_tree(rng, x, y, w // 2, h, pic_w, pic_h, min_size, out, leaf_bias, cout, cd)
            _split_tree(rng, x + w // 2, y, w // 2, h, pic_w, pic_h, min_size, out, leaf_bias, cout, cd)
            return
        if cross_y and h > min_size:
            cd = chroma_at(min(w, h // 2))
            _split_tree(rng, x, y, w, h // 2, pic_w, pic_h, min_size, out, leaf_bias, cout, cd)
            _split_tree(rng, x, y + h // 2, w, h // 2, pic_w, pic_h, min_size, out, leaf_bias, cout, cd)
            return
    opts = ["leaf"]
    if w == h and w > min_size:
        opts.append("qt")
    if w > min_size:
        opts.append("bv")
    if h > min_size:
        opts.append("bh")
    if w >= 4 * min_size:
        opts.append("tv")
    if h >= 4 * min_size:
        opts.append("th")
    p_leaf = leaf_bias if w * h <= 256 else leaf_bias / 3
    if w > 64 or h > 64:
        p_leaf = 0.0
    if len(opts) == 1 or rng.random() < p_leaf:
        out.append((x, y, w, h))
        if cout is not None and not chroma_done:
            cout.append((x, y, w, h))
        return
    kind = opts[1 + int(rng.integers(0, len(opts) - 1))]
    parts = {"qt": [(0, 0, w // 2, h // 2), (w // 2, 0, w // 2, h // 2), (0, h // 2, w // 2, h // 2),
                    (w // 2, h // 2, w // 2, h // 2)],
             "bv": [(0, 0, w // 2, h), (w // 2, 0, w // 2, h)],
             "bh": [(0, 0, w, h // 2), (0, h // 2, w, h // 2)],
             "tv": [(0, 0, w // 4, h), (w // 4, 0, w // 2, h), (3 * w // 4, 0, w // 4, h)],
             "th": [(0, 0, w, h // 4), (0, h // 4, w, h // 2), (0, 3 * h // 4, w, h // 4)]}[kind]
    cd = chroma_at(min(min(pw, ph) for _, _, pw, ph in parts))
    for dx, dy, pw, ph in parts:
        _split_tree(rng, x + dx, y + dy, pw, ph, pic_w, pic_h, min_size, out, leaf_bias, cout, cd)


def random_deblock_picture(vis_w, vis_h, ctu=32, bd=10, seed=0, dual_tree=False, isp_prob=0.25,
                           intra_prob=0.4, max_tb=64, leaf_bias=0.45):
    """A 4:2:0 picture with a random coding tree for the general decoder's
    deblocking: planes (Y, Cb, Cr) as uint16 arrays of the visible size with a
    per-transform-block DC step on smooth noise (so that edges take every
    filter decision), the luma cell map (DBK_CELL_DTYPE, one cell per 4x4 of
    the picture padded to whole CTUs), the chroma cell map (DBK_CCELL_DTYPE,
    one cell per 2x2 chroma samples) and slice parameters (DBK_PARAMS_DTYPE).
    The maps are what mark_tu (decode_general.rs:4837-4907) leaves: luma
    transform blocks tile each CU (max_tb, or ISP's 2 or 4 sub-partitions of
    1..64 samples), chroma ones each chroma CU of the same tree, or of a
    separate tree when dual_tree."""
    from . import DBK_CCELL_DTYPE, DBK_CELL_DTYPE, DBK_CBF, DBK_CODED, DBK_INTRA, DBK_NO_TU, DBK_PARAMS_DTYPE

    rng = np.random.default_rng(seed)
    pic_w, pic_h = -(-vis_w // ctu) * ctu, -(-vis_h // ctu) * ctu
    cols, rows = pic_w // 4, pic_h // 4
    ccols, crows = -(-(pic_w // 2) // 2), -(-(pic_h // 2) // 2)
    cells = np.zeros((rows, cols), DBK_CELL_DTYPE)
    cells["tu_id"] = DBK_NO_TU
    cells["ref_idx"] = -1
    cc = np.zeros((crows, ccols), DBK_CCELL_DTYPE)
    cc["tu_cb"] = DBK_NO_TU
    cc["tu_cr"] = DBK_NO_TU
    maxv = (1 << bd) - 1
    amp = 1 << (bd - 8)
    y_dc = np.zeros((pic_h, pic_w), np.int32)
    c_dc = [np.zeros((pic_h // 2, pic_w // 2), np.int32) for _ in range(2)]
    next_id = [0]

    def mark(comp, x, y, w, h, cbf):
        tid = next_id[0]
        next_id[0] += 1
        if comp == 0:
            x1, y1 = min(x + w, cols * 4), min(y + h, rows * 4)
            cx0, cx1, cy0, cy1 = x // 4, (x1 + 3) // 4, y // 4, (y1 + 3) // 4
            sub = cells[cy0:cy1, cx0:cx1]
            sub["tu_id"], sub["tu_w"], sub["tu_h"] = tid, w, h
            sub["flags"] = (sub["flags"] & (0xFF ^ DBK_CBF)) | (DBK_CBF if cbf else 0)
            y_dc[y:y + h, x:x + w] = int(rng.integers(-10, 11)) * amp
        else:
            cx, cy, cw_, ch_ = x // 2, y // 2, w // 2, h // 2
            x1, y1 = min(cx + cw_, ccols * 2), min(cy + ch_, crows * 2)
            sub = cc[cy // 2:(y1 + 1) // 2, cx // 2:(x1 + 1) // 2]
            sub["tu_cb" if comp == 1 else "tu_cr"] = tid
            sub["tu_w"], sub["tu_h"] = cw_, ch_
            c_dc[comp - 1][cy:cy + ch_, cx:cx + cw_] = int(rng.integers(-8, 9)) * amp

    cus, shared_ccus = [], []
    for ty in range(0, pic_h, ctu):
        for tx in range(0, pic_w, ctu):
            _split_tree(rng, tx, ty, ctu, ctu, vis_w, vis_h, 4, cus, leaf_bias, shared_ccus)
    for (x, y, w, h) in cus:
        intra = rng.random() < intra_prob
        sub = cells[y // 4:(y + h + 3) // 4, x // 4:(x + w + 3) // 4]
        sub["flags"] = DBK_CODED | (DBK_INTRA if intra else 0)
        if not intra:
            d = int(rng.integers(1, 4))
            for l in range(2):
                if d & (1 << l):
                    sub["ref_idx"][..., l] = int(rng.integers(0, 3))
                    big = rng.random() < 0.5
                    sub["mv"][..., l, :] = rng.integers(-40, 41, 2) if big else rng.integers(-3, 4, 2)
        if intra and rng.random() < isp_prob and w * h > 16 and (w < 64 or h < 64):
            vert = bool(rng.integers(0, 2)) if w > 1 and h > 1 else False
            n = 2 if (w, h) in ((4, 8), (8, 4)) else 4
            for i in range(n):
                if vert:
                    mark(0, x + i * (w // n), y, w // n, h, rng.random() < 0.6)
                else:
                    mark(0, x, y + i * (h // n), w, h // n, rng.random() < 0.6)
        else:
            tb = min(max_tb, 64)
            for yy in range(y, y + h, min(h, tb)):
                for xx in range(x, x + w, min(w, tb)):
                    mark(0, xx, yy, min(w, tb), min(h, tb), rng.random() < 0.6)
    ccus = []
    if dual_tree:
        for ty in range(0, pic_h, ctu):
            for tx in range(0, pic_w, ctu):
                _split_tree(rng, tx, ty, ctu, ctu, vis_w, vis_h, 8, ccus, leaf_bias)
    else:
        ccus = shared_ccus
    for (x, y, w, h) in ccus:
        tb = 64
        for yy in range(y, y + h, min(h, tb)):
            for xx in range(x, x + w, min(w, tb)):
                for comp in (1, 2):
                    mark(comp, xx, yy, min(w, tb), min(h, tb), True)
    # smooth content plus the per-block steps
    yn, un, vn = value_noise_frame(pic_w, pic_h, 10, frame=seed)

    def scale(p):
        return p.astype(np.int32) << (bd - 10) if bd >= 10 else p.astype(np.int32) >> (10 - bd)

    ys = np.clip(scale(yn) // 4 + (maxv // 3) + y_dc + rng.integers(-amp, amp + 1, y_dc.shape), 0, maxv)
    us = np.clip(scale(un) // 4 + (maxv // 3) + c_dc[0] + rng.integers(-amp, amp + 1, c_dc[0].shape), 0, maxv)
    vs = np.clip(scale(vn) // 4 + (maxv // 3) + c_dc[1] + rng.integers(-amp, amp + 1, c_dc[1].shape), 0, maxv)
    cw, ch = (vis_w + 1) // 2, (vis_h + 1) // 2
    planes = (ys[:vis_h, :vis_w].astype(np.uint16), us[:ch, :cw].astype(np.uint16), vs[:ch, :cw].astype(np.uint16))
    params = np.zeros((), DBK_PARAMS_DTYPE)
    qp = int(rng.integers(22, 46))
    params["qp"] = [qp, qp + int(rng.integers(-3, 2)), qp + int(rng.integers(-3, 2))]
    params["beta_offset_div2"] = rng.integers(-4, 5, 3)
    params["tc_offset_div2"] = rng.integers(-4, 5, 3)
    params["num_ref"] = [3, 2]
    params["ref_poc"] = rng.integers(-8, 9, (2, 16))
    return planes, cells, cc, params


def random_gen_intra_state(width, height, bd=10, seed=0, hole_prob=0.15):
    """Planes and decoded maps for the general decoder's intra prediction:
    smooth content with noise (Y at width x height, Cb / Cr at half), and
    decoded maps that are the raster-order decode of a random position
    (everything above it and left of it on its CTU row band) with random
    holes; one byte per 4x4 luma cell, one per chroma sample."""
    rng = np.random.default_rng(seed)
    maxv = (1 << bd) - 1
    y, u, v = value_noise_frame(max(width, 128), max(height, 128), 10, frame=seed)
    sc = (lambda p: (p.astype(np.int32) << (bd - 10)) if bd >= 10 else (p.astype(np.int32) >> (10 - bd)))
    Y = np.clip(sc(y[:height, :width]) + rng.integers(-3, 4, (height, width)), 0, maxv).astype(np.uint16)
    U = np.clip(sc(u[:height // 2, :width // 2]) + rng.integers(-3, 4, (height // 2, width // 2)), 0, maxv).astype(np.uint16)
    V = np.clip(sc(v[:height // 2, :width // 2]) + rng.integers(-3, 4, (height // 2, width // 2)), 0, maxv).astype(np.uint16)
    cy, cx = rng.integers(0, height), rng.integers(0, width)
    yy, xx = np.mgrid[0:height // 4, 0:width // 4]
    dec_y = ((yy * 4 < cy - 32) | ((yy * 4 < cy + 32) & (xx * 4 < cx))).astype(np.uint8)
    dec_y &= (rng.random(dec_y.shape) >= hole_prob).astype(np.uint8)
    yc, xc = np.mgrid[0:height // 2, 0:width // 2]
    dec_c = ((yc * 2 < cy - 32) | ((yc * 2 < cy + 32) & (xc * 2 < cx))).astype(np.uint8)
    dec_c &= (rng.random(dec_c.shape) >= hole_prob / 4).astype(np.uint8)
    return (Y, U, V), dec_y, dec_c


def random_gen_intra_reqs(width, height, n, seed=0):
    """Random requests of every kind (GEN_INTRA_REQ_DTYPE) inside a width x
    height picture: luma blocks 4..64 with Planar / DC / angular (MRL 0..2),
    BDPCM, ISP sub-partitions of 4..64-sample CUs (1..64 samples, including
    the narrow vertical ones that share a 4-wide region), and chroma blocks
    2..32 with Planar / DC / angular / CCLM."""
    from . import GEN_INTRA_REQ_DTYPE

    rng = np.random.default_rng(seed)
    r = np.zeros(n, GEN_INTRA_REQ_DTYPE)
    off = 0
    for i in range(n):
        q = r[i]
        kind = int(rng.integers(0, 6))
        if kind <= 2:  # luma regular / MRL / BDPCM
            w, h = 1 << int(rng.integers(2, 7)), 1 << int(rng.integers(2, 7))
            x = int(rng.integers(0, (width - w) // 4 + 1)) * 4
            y = int(rng.integers(0, (height - h) // 4 + 1)) * 4
            q["comp"], q["x"], q["y"], q["w"], q["h"] = 0, x, y, w, h
            q["cu_x"], q["cu_y"], q["cu_w"], q["cu_h"] = x, y, w, h
            q["mode"] = int(rng.integers(0, 67))
            if kind == 1:
                q["mrl"] = int(rng.integers(1, 3))
            if kind == 2:
                q["bdpcm"] = int(rng.integers(1, 3))
        elif kind == 3:  # ISP sub-partition
            cw, ch = 1 << int(rng.integers(2, 7)), 1 << int(rng.integers(2, 7))
            cx = int(rng.integers(0, (width - cw) // 4 + 1)) * 4
            cy = int(rng.integers(0, (height - ch) // 4 + 1)) * 4
            ver = bool(rng.integers(0, 2))
            nparts = 2 if (cw, ch) in ((4, 8), (8, 4)) else 4
            k = int(rng.integers(0, nparts))
            if ver:
                w, h = max(1, cw // nparts), ch
                x, y = cx + k * w, cy
            else:
                w, h = cw, max(1, ch // nparts)
                x, y = cx, cy + k * h
            q["comp"], q["x"], q["y"], q["w"], q["h"] = 0, x, y, w, h
            q["cu_x"], q["cu_y"], q["cu_w"], q["cu_h"] = cx, cy, cw, ch
            q["isp"] = 2 if ver else 1
            q["mode"] = int(rng.integers(0, 67))
        else:  # chroma
            w, h = 1 << int(rng.integers(1, 6)), 1 << int(rng.integers(1, 6))
            x = int(rng.integers(0, (width // 2 - w) // 2 + 1)) * 2
            y = int(rng.integers(0, (height // 2 - h) // 2 + 1)) * 2
            q["comp"], q["x"], q["y"], q["w"], q["h"] = int(rng.integers(1, 3)), x, y, w, h
            q["mode"] = int(rng.choice([0, 1, int(rng.integers(2, 67)), 81, 82, 83]))
        q["out_off"] = off
        off += int(q["w"]) * int(q["h"])
    return r, off


# ------------------------------------------------------------------ encoded content --
# The full-frame configuration decodes what the repo's own encoder makes of
# its content: value-noise frames encoded all-intra (the reference encodes
# every 10-bit frame as an IDR, mod.rs:1727-1802) with the frame path's
# tools, then decoded with deblocking, SAO and ALF (SAO / ALF parameters
# are seeded per CTU: the reference encoders never switch them on,
# slice.rs:2611-2630).

ENC_TOOLS = TOOL_ENC_FULL_INTRA | TOOL_ENC_CCLM | TOOL_DEP_QUANT | TOOL_DEBLOCK
DEC_TOOLS = TOOL_DEP_QUANT | TOOL_DEBLOCK | TOOL_SAO | TOOL_ALF


def chroma_qp_scaled(qp, bd):
    """Qp'C of derived_chroma_qp_bd (hls.rs:796-802) with a zero chroma QP offset."""
    off = 6 * (bd - 8)
    qpi = min(63, max(-off, qp))
    mapped = qpi if qpi <= 26 else qpi - 1
    return min(63 + off, max(0, min(63, max(-off, mapped)) + off))


def workload_picture(index, frames_per_qp, qps, width=1920, height=1080, bd=10, ctu_log2=5):
    """(frame, qp, PIC_DTYPE encoder descriptor) of picture `index` of a
    workload of frames_per_qp frames at each QP, QP-major; the coded height
    is the CTU multiple above the visible one (mod.rs:300-324)."""
    ctu = 1 << ctu_log2
    frame, qp = index % frames_per_qp, qps[index // frames_per_qp]
    p = np.zeros((), PIC_DTYPE)
    p["width"], p["height"] = -(-width // ctu) * ctu, -(-height // ctu) * ctu
    p["visible_width"], p["visible_height"] = width, height
    p["bit_depth"], p["chroma_format"], p["ctu_log2"] = bd, 1, ctu_log2
    p["slice_qp"], p["chroma_qp_scaled"] = qp, chroma_qp_scaled(qp, bd)
    p["tools"] = ENC_TOOLS
    p["alf_aps"] = -1
    return frame, qp, p


def workload_sources(frame, p, stream=0):
    """Coded-size source planes of frame `frame` of content stream `stream`
    (4:2:0, the picture's bit depth; edge padding below the visible rows)."""
    w, h, vw, vh = int(p["width"]), int(p["height"]), int(p["visible_width"]), int(p["visible_height"])
    bd = int(p["bit_depth"])
    y, u, v = value_noise_frame(vw, vh, 10, frame=frame, stream=stream)
    if bd != 10:
        y, u, v = ((a.astype(np.int32) << bd >> 10).astype(np.uint16) if bd > 10 else (a >> (10 - bd))
                   for a in (y, u, v))
    cw, ch = chroma_dims(w, h, 1)
    return pad_to(y, w, h), pad_to(u, cw, ch), pad_to(v, cw, ch)


def compact_levels(p, cus, levels):
    """The picture's coded TBs' levels in CU order (luma, Cb, Cr of each CU),
    as a parser emits them; returns (cus with new offsets, levels)."""
    cf = int(p["chroma_format"])
    tb = min(1 << int(p["ctu_log2"]), 32)
    cw, ch = chroma_dims(tb, tb, cf)
    sizes = np.array([tb * tb, max(cw, 2) * max(ch, 2) if cf else 0, max(cw, 2) * max(ch, 2) if cf else 0])
    cus = cus.copy()
    lo = cus["level_off"].astype(np.int64)
    coded = ((cus["cbf"][:, None] >> np.arange(3)) & 1).astype(bool) & (lo >= 0)
    if not cf:
        coded[:, 1:] = False
    n = coded * sizes[None, :]
    new = (np.cumsum(n.ravel()) - n.ravel()).reshape(n.shape)
    out = np.zeros(int(n.sum()), np.int16)
    for c in range(3):
        k = np.nonzero(coded[:, c])[0]
        if len(k):
            ar = np.arange(sizes[c])[None, :]
            out[new[k, c][:, None] + ar] = levels[lo[k, c][:, None] + ar]
    cus["level_off"] = np.where(coded, new, -1).astype(np.int32)
    return cus, out


def _tb_sizes(p):
    """Levels per TB of a frame-path picture: (luma, Cb, Cr)."""
    cf = int(p["chroma_format"])
    tb = min(1 << int(p["ctu_log2"]), 32)
    cw, ch = chroma_dims(tb, tb, cf)
    nc = max(cw, 2) * max(ch, 2) if cf else 0
    return tb, (tb * tb, nc, nc)


def sparsify(pics, cus, levels):
    """The batch with every picture's TBs in the sparse level form
    (TOOL_SPARSE_LEVELS): per coded TB, at an even offset, the count of its
    nonzero levels, one unused word, then (raster index, level) int16 pairs
    with rising indices. Returns (pics, cus, levels); the inputs are not
    changed."""
    pics = np.array(pics, PIC_DTYPE, copy=True)
    cus = np.array(cus, CU_DTYPE, copy=True)
    levels = np.asarray(levels, np.int16)
    lo = cus["level_off"].astype(np.int64)
    new_off = np.full(lo.shape, -1, np.int64)
    blocks, at = [], 0
    for i in range(len(pics)):
        p = pics[i]
        tb, sizes = _tb_sizes(p)
        c0 = int(p["cu_offset"])
        ncu = (int(p["width"]) // tb) * (int(p["height"]) // tb)
        cbf = cus["cbf"][c0:c0 + ncu]
        for c in range(3 if int(p["chroma_format"]) else 1):
            coded = ((cbf >> c) & 1).astype(bool) & (lo[c0:c0 + ncu, c] >= 0)
            k = np.nonzero(coded)[0]
            if not len(k):
                continue
            g = levels[lo[c0 + k, c][:, None] + np.arange(sizes[c])[None, :]]
            nz = g != 0
            cnt = nz.sum(1)
            words = 2 + 2 * cnt
            start = np.cumsum(words) - words
            blk = np.zeros(int(words.sum()), np.int16)
            blk[start] = cnt
            r, col = np.nonzero(nz)
            rank = np.arange(len(r)) - (np.cumsum(cnt) - cnt)[r]
            at_e = start[r] + 2 + 2 * rank
            blk[at_e] = col
            blk[at_e + 1] = g[r, col]
            new_off[c0 + k, c] = at + start
            blocks.append(blk)
            at += len(blk)
        pics["tools"][i] = int(p["tools"]) | TOOL_SPARSE_LEVELS
    if at >= 1 << 31:
        raise ValueError("sparse level pool exceeds int32 offsets")
    cus["level_off"] = new_off.astype(np.int32)
    return pics, cus, np.concatenate(blocks) if blocks else np.zeros(0, np.int16)


def densify(pics, cus, levels):
    """The inverse of sparsify: raster-order TBs, TOOL_SPARSE_LEVELS cleared."""
    pics = np.array(pics, PIC_DTYPE, copy=True)
    cus = np.array(cus, CU_DTYPE, copy=True)
    levels = np.asarray(levels, np.int16)
    lo = cus["level_off"].astype(np.int64)
    new_off = np.full(lo.shape, -1, np.int64)
    out, at = [], 0
    for i in range(len(pics)):
        p = pics[i]
        tb, sizes = _tb_sizes(p)
        c0 = int(p["cu_offset"])
        ncu = (int(p["width"]) // tb) * (int(p["height"]) // tb)
        for k in range(ncu):
            for c in range(3 if int(p["chroma_format"]) else 1):
                o = int(lo[c0 + k, c])
                if o < 0 or not (int(cus["cbf"][c0 + k]) >> c) & 1:
                    continue
                tbl = np.zeros(sizes[c], np.int16)
                n = int(levels[o])
                pairs = levels[o + 2:o + 2 + 2 * n].reshape(-1, 2)
                tbl[pairs[:, 0].astype(np.int64)] = pairs[:, 1]
                new_off[c0 + k, c] = at
                out.append(tbl)
                at += sizes[c]
        pics["tools"][i] = int(p["tools"]) & ~TOOL_SPARSE_LEVELS
    cus["level_off"] = new_off.astype(np.int32)
    return pics, cus, np.concatenate(out) if out else np.zeros(0, np.int16)


def decoder_picture(index, p_enc, cus, levels, seed):
    """Decoder records of one encoded picture: the encoder's CUs with a
    compact level pool, DEC_TOOLS, and per-CTU SAO / ALF parameters seeded
    by (seed, index). Returns (pic, cus, levels, ctus)."""
    p = np.asarray(p_enc, PIC_DTYPE).copy()
    cus, levels = compact_levels(p, cus, levels)
    p["tools"] = DEC_TOOLS
    p["alf_aps"] = 0
    ctu = 1 << int(p["ctu_log2"])
    rng = np.random.default_rng([seed, index])
    ctus = random_ctu_params(rng, int(p["width"]), int(p["height"]), ctu, int(p["bit_depth"]),
                             int(p["chroma_format"]))
    return p, cus, levels, ctus


def workload_aps(seed):
    """The workload's ALF APS (fixed-filter coefficient sets, seeded)."""
    return synthetic_aps(np.random.default_rng([seed, 1 << 30]))


def assemble(parts, aps):
    """One batch from per-picture (pic, cus, levels, ctus) parts: offsets
    rebased into shared record and level arrays. Returns (pics, cus, levels,
    ctus, aps)."""
    pics, cu_l, lv_l, ctu_l = [], [], [], []
    n_cu = n_lv = n_ctu = 0
    for p, cus, levels, ctus in parts:
        p = np.asarray(p, PIC_DTYPE).copy()
        p["cu_offset"], p["ctu_offset"] = n_cu, n_ctu
        cus = cus.copy()
        cus["level_off"] = np.where(cus["level_off"] >= 0, cus["level_off"] + n_lv, -1)
        pics.append(p)
        cu_l.append(cus)
        lv_l.append(levels)
        ctu_l.append(ctus)
        n_cu += len(cus)
        n_lv += len(levels)
        n_ctu += len(ctus)
    return (np.array(pics, PIC_DTYPE), np.concatenate(cu_l), np.concatenate(lv_l), np.concatenate(ctu_l),
            aps)


def encoded_workload(ctx, frames_per_qp, qps, seed, sources=None, width=1920, height=1080, bd=10,
                     encode_chunk=32, stream=0):
    """The decoder records of frames_per_qp value-noise frames at each QP,
    encoded on the GPU by `ctx` (vvcg_encode_batch, the frame-path encoder;
    bit-exact with the oracle's encoder). `sources` maps a frame index to its
    coded-size planes (generated here when absent). Returns (pics, cus,
    levels, ctus, aps) ready for Batch."""
    parts = encoded_parts(ctx, frames_per_qp, qps, seed, sources, width, height, bd, encode_chunk, stream)
    return assemble(parts, workload_aps(seed))


def encoded_parts(ctx, frames_per_qp, qps, seed, sources=None, width=1920, height=1080, bd=10, encode_chunk=32,
                  stream=0):
    """encoded_workload's per-picture (pic, cus, levels, ctus) parts."""
    n = frames_per_qp * len(qps)
    descs = [workload_picture(i, frames_per_qp, qps, width, height, bd) for i in range(n)]
    src = dict(sources or {})
    for f, _, p in descs:
        if f not in src:
            src[f] = workload_sources(f, p, stream)
    parts = []
    for a in range(0, n, encode_chunk):
        chunk = descs[a:a + encode_chunk]
        pics = np.array([p for _, _, p in chunk], PIC_DTYPE)
        cus, levels = ctx.encode_batch(pics, [src[f] for f, _, _ in chunk])
        # the encoder's pictures are consecutive in its records
        tb = min(1 << int(pics[0]["ctu_log2"]), 32)
        at = 0
        for j, (_, _, p) in enumerate(chunk):
            ncu = (int(p["width"]) // tb) * (int(p["height"]) // tb)
            parts.append(decoder_picture(a + j, p, cus[at:at + ncu], levels, seed))
            at += ncu
    return parts


def oracle_workload_picture(oracle, index, frames_per_qp, qps, seed, width=1920, height=1080, bd=10, stream=0):
    """The same decoder records for one picture, encoded by the oracle's
    encoder on the CPU (for the CPU baseline, which runs without a GPU)."""
    f, _, p = workload_picture(index, frames_per_qp, qps, width, height, bd)
    y, u, v = workload_sources(f, p, stream)
    t = int(p["tools"])
    opts = ((oracle.OPT_FULL_INTRA if t & TOOL_ENC_FULL_INTRA else 0) | (oracle.OPT_CCLM if t & TOOL_ENC_CCLM else 0)
            | (oracle.OPT_DEP_QUANT if t & TOOL_DEP_QUANT else 0) | (oracle.OPT_DEBLOCK if t & TOOL_DEBLOCK else 0))
    cus, levels, _ = oracle.encode_frame(y, u, v, int(p["bit_depth"]), int(p["slice_qp"]), int(p["ctu_log2"]),
                                         opts, int(p["chroma_format"]))
    return decoder_picture(index, p, cus, levels, seed)


# ------------------------------------------------------------------ batching --
# The batching configuration: independent streams of uneven resolution and
# bit depth decoded in one pass.
BATCH_RESOLUTIONS = ((416, 240), (832, 480), (1280, 720), (1920, 1080), (3840, 2160))
BATCH_WEIGHTS = (0.3, 0.3, 0.2, 0.15, 0.05)


def batching_streams(n_streams, seed):
    """(width, height, bit depth, QP) of each stream: resolution drawn with
    BATCH_WEIGHTS, bit depth uniform over {8, 10}, QP uniform in 22..37."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_streams):
        w, h = BATCH_RESOLUTIONS[int(rng.choice(len(BATCH_RESOLUTIONS), p=BATCH_WEIGHTS))]
        out.append((w, h, int(rng.choice((8, 10))), int(rng.integers(22, 38))))
    return out


# ---------------------------------------------------------------------------
# General-decoder intra pictures (coding trees of 4x4..128x128 blocks)
# ---------------------------------------------------------------------------

def random_alf_general_params(rng):
    """An ALF_PARAMS_DTYPE record with random luma, chroma and CCALF filters."""
    from . import ALF_PARAMS_DTYPE

    a = np.zeros((), ALF_PARAMS_DTYPE)
    a["num_luma_filters"] = int(rng.integers(1, 26))
    a["luma_clip"] = int(rng.integers(0, 2))
    a["coeff_delta_idx"] = rng.integers(0, int(a["num_luma_filters"]), 25)
    a["luma_coeff"] = rng.integers(-40, 41, (25, 12))
    a["luma_clip_idx"] = rng.integers(0, 4, (25, 12))
    a["num_chroma_filters"] = int(rng.integers(1, 9))
    a["chroma_clip"] = int(rng.integers(0, 2))
    a["chroma_coeff"] = rng.integers(-40, 41, (8, 6))
    a["chroma_clip_idx"] = rng.integers(0, 4, (8, 6))
    a["num_cc_cb"], a["num_cc_cr"] = int(rng.integers(1, 5)), int(rng.integers(0, 5))
    a["cc_cb"] = rng.integers(-64, 65, (4, 7))
    a["cc_cr"] = rng.integers(-64, 65, (4, 7))
    return a


def _general_groups(rng, tx, ty, ctu, vis_w, vis_h, leaf_bias, out):
    """The coding units of one CTU in decode order as groups: ("cu", x, y, w,
    h, with_chroma) for a coding unit (with its chroma when its node is at
    least 8x8 luma) and ("chroma", x, y, w, h) for the chroma of a node whose
    luma children are narrower or shorter than 8, after its last child.
    The same splitting rules as _split_tree (implicit halving across the
    picture edge, no leaf above 64)."""

    def walk(x, y, w, h, chroma_done):
        if x >= vis_w or y >= vis_h:
            return
        cross_x, cross_y = x + w > vis_w, y + h > vis_h
        parts = None
        if cross_x or cross_y:
            if cross_x and cross_y and w > 4 and h > 4:
                parts = [(0, 0, w // 2, h // 2), (w // 2, 0, w // 2, h // 2), (0, h // 2, w // 2, h // 2),
                         (w // 2, h // 2, w // 2, h // 2)]
            elif cross_x and w > 4:
                parts = [(0, 0, w // 2, h), (w // 2, 0, w // 2, h)]
            elif cross_y and h > 4:
                parts = [(0, 0, w, h // 2), (0, h // 2, w, h // 2)]
        if parts is None:
            opts = ["leaf"]
            if w == h and w > 4:
                opts.append("qt")
            if w > 4:
                opts.append("bv")
            if h > 4:
                opts.append("bh")
            if w >= 16:
                opts.append("tv")
            if h >= 16:
                opts.append("th")
            p_leaf = leaf_bias if w * h <= 256 else leaf_bias / 3
            if w > 64 or h > 64:
                p_leaf = 0.0
            if len(opts) == 1 or rng.random() < p_leaf:
                out.append(("cu", x, y, w, h, not chroma_done))
                return
            kind = opts[1 + int(rng.integers(0, len(opts) - 1))]
            parts = {"qt": [(0, 0, w // 2, h // 2), (w // 2, 0, w // 2, h // 2), (0, h // 2, w // 2, h // 2),
                            (w // 2, h // 2, w // 2, h // 2)],
                     "bv": [(0, 0, w // 2, h), (w // 2, 0, w // 2, h)],
                     "bh": [(0, 0, w, h // 2), (0, h // 2, w, h // 2)],
                     "tv": [(0, 0, w // 4, h), (w // 4, 0, w // 2, h), (3 * w // 4, 0, w // 4, h)],
                     "th": [(0, 0, w, h // 4), (0, h // 4, w, h // 2), (0, 3 * h // 4, w, h // 4)]}[kind]
        here = not chroma_done and min(min(pw, ph) for _, _, pw, ph in parts) < 8
        for dx, dy, pw, ph in parts:
            walk(x + dx, y + dy, pw, ph, chroma_done or here)
        if here:
            out.append(("chroma", x, y, w, h))

    walk(tx, ty, ctu, ctu, False)


def random_general_picture(vis_w, vis_h, ctu=64, bd=10, qp=32, seed=0, tools=TOOL_DEBLOCK | TOOL_SAO | TOOL_ALF,
                           dep_quant=False, isp_prob=0.2, mrl_prob=0.2, bdpcm_prob=0.08, lfnst_prob=0.15,
                           mts_prob=0.2, ts_prob=0.08, coded_prob=0.75, leaf_bias=0.45, implicit_mts=True):
    """One general-decoder intra picture as GenBatch parts: (pic, tbs,
    group_sizes, levels, slot_count, sao, alf_ctus, alf_params). Blocks are
    in decode order with slots and level offsets local to the picture."""
    from . import (GEN_PIC_DTYPE, GEN_TB_DTYPE, SAO_DTYPE, ALF_CTU_DTYPE, ISP_HOR, ISP_VER, TU_DEP_QUANT,
                   TU_TRANSFORM_SKIP, TU_BDPCM_HOR, TU_BDPCM_VER, TU_IMPLICIT_MTS)

    rng = np.random.default_rng(seed)
    pic_w, pic_h = -(-vis_w // ctu) * ctu, -(-vis_h // ctu) * ctu
    groups = []
    for ty in range(0, pic_h, ctu):
        for tx in range(0, pic_w, ctu):
            _general_groups(rng, tx, ty, ctu, vis_w, vis_h, leaf_bias, groups)
    lqp = min(63 + 6 * (bd - 8), qp + 6 * (bd - 8))
    cqp = chroma_qp_scaled(qp, bd)
    tbs, sizes, lv_chunks = [], [], []
    slot = lvl = 0

    def add(x, y, w, h, cu, comp, mode, mrl=0, isp=0, bdpcm=0, ts=False, mts=0, lfnst=0, coded=True):
        nonlocal slot, lvl
        t = np.zeros((), GEN_TB_DTYPE)
        t["pred"]["x"], t["pred"]["y"], t["pred"]["w"], t["pred"]["h"] = x, y, w, h
        t["pred"]["cu_x"], t["pred"]["cu_y"], t["pred"]["cu_w"], t["pred"]["cu_h"] = cu
        t["pred"]["comp"], t["pred"]["mode"], t["pred"]["mrl"] = comp, mode, mrl
        t["pred"]["isp"], t["pred"]["bdpcm"] = isp, bdpcm
        t["pred"]["out_off"] = slot
        tu = t["tu"]
        tu["log2_w"], tu["log2_h"] = int(w).bit_length() - 1, int(h).bit_length() - 1
        tu["bit_depth"], tu["qp"] = bd, lqp if comp == 0 else cqp
        flags = 0
        if ts:
            flags |= TU_TRANSFORM_SKIP
            if bdpcm:
                flags |= TU_BDPCM_HOR if bdpcm == 1 else TU_BDPCM_VER
        elif dep_quant:
            flags |= TU_DEP_QUANT
        if comp == 0 and implicit_mts and not isp and not ts and mts == 0 and lfnst == 0:
            flags |= TU_IMPLICIT_MTS
        tu["flags"], tu["mts_idx"], tu["lfnst_idx"], tu["lfnst_mode"] = flags, mts, lfnst, mode if lfnst else 0
        tu["out_off"] = slot
        if coded:
            tu["in_off"] = lvl
            lv = _tb_levels(rng, 1, w, h, int(tu["qp"]))[0]
            if lfnst:  # LFNST codes only its top-left coefficients
                keep = np.zeros_like(lv)
                keep[:4, :4] = lv[:4, :4]
                lv = keep if keep.any() else np.pad(np.ones((1, 1), np.int16), ((0, h - 1), (0, w - 1)))
            if mts and (w == 32 or h == 32):
                lv[16:, :] = 0
                lv[:, 16:] = 0
            lv_chunks.append(lv.reshape(-1))
            lvl += w * h
        t["coded"] = 1 if coded else 0
        tbs.append(t)
        slot += w * h

    for g in groups:
        n0 = len(tbs)
        if g[0] == "cu":
            _, x, y, w, h, with_chroma = g
            mode = int(rng.integers(0, 67))
            isp = mrl = bdpcm = 0
            if w * h > 16 and w <= 64 and h <= 64 and rng.random() < isp_prob:
                isp = ISP_HOR if rng.random() < 0.5 else ISP_VER
            elif w <= 32 and h <= 32 and rng.random() < bdpcm_prob:
                bdpcm = 1 + int(rng.integers(0, 2))
                mode = 18 if bdpcm == 1 else 50
            elif y % ctu and w >= 4 and h >= 4 and rng.random() < mrl_prob:
                mrl = 1 + int(rng.integers(0, 2))
            cu = (x, y, w, h)
            if isp:
                n = 2 if (w, h) in ((4, 8), (8, 4)) else 4
                for k in range(n):
                    sx, sy, sw, sh = (x, y + k * h // n, w, h // n) if isp == ISP_HOR else (x + k * w // n, y, w // n, h)
                    add(sx, sy, sw, sh, cu, 0, mode, isp=isp, coded=rng.random() < coded_prob)
            else:
                tb = 64
                for yy in range(y, y + h, min(h, tb)):
                    for xx in range(x, x + w, min(w, tb)):
                        tw, th = min(w, tb), min(h, tb)
                        ts = bool(bdpcm) or (tw <= 32 and th <= 32 and rng.random() < ts_prob)
                        lfnst = 0
                        mts = 0
                        if not ts and tw == th and tw >= 4 and rng.random() < lfnst_prob:
                            lfnst = 1 + int(rng.integers(0, 2))
                        elif not ts and tw <= 32 and th <= 32 and tw >= 4 and th >= 4 and rng.random() < mts_prob:
                            mts = 1 + int(rng.integers(0, 4))
                        add(xx, yy, tw, th, cu, 0, mode, mrl=mrl, bdpcm=bdpcm, ts=ts, mts=mts, lfnst=lfnst,
                            coded=bdpcm or rng.random() < coded_prob)
            if with_chroma:
                groups_chroma = [(x, y, w, h)]
            else:
                groups_chroma = []
        else:
            _, x, y, w, h = g
            groups_chroma = [(x, y, w, h)]
        for (x, y, w, h) in groups_chroma:
            cm = int(rng.choice([0, 1, 18, 50, 66, 81, 82, 83]))
            cw_, ch_ = w // 2, h // 2
            for yy in range(0, ch_, min(ch_, 32)):
                for xx in range(0, cw_, min(cw_, 32)):
                    tw, th = min(cw_, 32), min(ch_, 32)
                    for comp in (1, 2):
                        add(x // 2 + xx, y // 2 + yy, tw, th, (x, y, w, h), comp, cm,
                            ts=tw <= 32 and rng.random() < ts_prob, coded=rng.random() < coded_prob)
        sizes.append(len(tbs) - n0)
    cols, rows = -(-vis_w // ctu), -(-vis_h // ctu)
    nctu = cols * rows
    sao = np.zeros(3 * nctu, SAO_DTYPE)
    kind = rng.integers(0, 3, 3 * nctu)
    omax = (1 << (min(bd, 10) - 5)) - 1
    sao["type"] = kind
    sao["band_or_class"] = np.where(kind == 1, rng.integers(0, 32, 3 * nctu), rng.integers(0, 4, 3 * nctu))
    sao["offsets"] = np.where((kind == 2)[:, None],
                              rng.integers(0, omax + 1, (3 * nctu, 4)) * np.array([1, 1, -1, -1]),
                              rng.integers(-omax, omax + 1, (3 * nctu, 4)))
    alf = np.zeros(nctu, ALF_CTU_DTYPE)
    alf["luma_mode"] = rng.integers(0, 3, nctu)
    alf["luma_set"] = rng.integers(0, 16, nctu)
    alf["cb_alt"] = np.where(rng.random(nctu) < 0.7, rng.integers(0, 8, nctu), 0xFF)
    alf["cr_alt"] = np.where(rng.random(nctu) < 0.7, rng.integers(0, 8, nctu), 0xFF)
    alf["cc_cb"] = rng.integers(0, 5, nctu)
    alf["cc_cr"] = rng.integers(0, 5, nctu)
    p = np.zeros((), GEN_PIC_DTYPE)
    p["width"], p["height"], p["vis_width"], p["vis_height"] = pic_w, pic_h, vis_w, vis_h
    p["bit_depth"], p["ctu_log2"], p["vert_collocated"], p["tools"] = bd, int(ctu).bit_length() - 1, 0, tools
    p["alf_params"] = 0
    d = p["dbk"]
    d["qp"] = [qp, min(63, max(0, qp + int(rng.integers(-3, 2)))), min(63, max(0, qp + int(rng.integers(-3, 2))))]
    d["beta_offset_div2"] = rng.integers(-4, 5, 3)
    d["tc_offset_div2"] = rng.integers(-4, 5, 3)
    levels = np.concatenate(lv_chunks) if lv_chunks else np.zeros(0, np.int16)
    return (p, np.array(tbs, GEN_TB_DTYPE), np.array(sizes, np.uint32), levels, slot, sao, alf,
            random_alf_general_params(rng))


def general_batch(parts):
    """GenBatch inputs from random_general_picture parts: pictures, blocks,
    group_first, levels and slots rebased into shared arrays. Returns a dict
    of the GenBatch constructor's arguments."""
    from . import GEN_PIC_DTYPE

    pics, tbs, firsts, levels, saos, alfs, prms = [], [], [0], [], [], [], []
    n_tb = n_grp = n_lv = n_slot = n_sao = n_alf = 0
    for k, (p, t, sizes, lv, slots, sao, alf, prm) in enumerate(parts):
        p = np.asarray(p, GEN_PIC_DTYPE).copy()
        p["group_offset"], p["num_groups"] = n_grp, len(sizes)
        p["sao_offset"], p["alf_offset"], p["alf_params"] = n_sao, n_alf, k
        t = t.copy()
        t["pred"]["out_off"] += n_slot
        t["tu"]["out_off"] += n_slot
        t["tu"]["in_off"] = np.where(t["coded"] != 0, t["tu"]["in_off"] + n_lv, 0)
        pics.append(p)
        tbs.append(t)
        firsts.extend((n_tb + np.cumsum(sizes)).tolist())
        levels.append(lv)
        saos.append(sao)
        alfs.append(alf)
        prms.append(prm)
        n_tb += len(t)
        n_grp += len(sizes)
        n_lv += len(lv)
        n_slot += slots
        n_sao += len(sao)
        n_alf += len(alf)
    return dict(pics=np.array(pics, GEN_PIC_DTYPE), tbs=np.concatenate(tbs), group_first=np.array(firsts, np.uint32),
                levels=np.concatenate(levels), slot_count=n_slot, sao=np.concatenate(saos),
                alf_ctus=np.concatenate(alfs), alf_params=np.array(prms))
