"""GPU parity: the frame-path encoder (vvcg_encode_batch) against the oracle's
restatement of slice::encode_vvc_frame_picture, bit-exact: the same modes,
cbfs and levels per TB and the same reconstruction; and the closed loop the
reference's round-trip tests use (decoding the emitted records gives the
encoder's reconstruction)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

OPT_FULL, OPT_CCLM, OPT_DQ, OPT_DBF = 1, 2, 4, 8


def _desc(pkg, w, h, bd, qp, ctu_log2, opts, cf, vis=None):
    p = np.zeros((), pkg.PIC_DTYPE)
    p["width"], p["height"] = w, h
    p["visible_width"], p["visible_height"] = vis or (w, h)
    p["bit_depth"], p["chroma_format"], p["ctu_log2"] = bd, cf, ctu_log2
    p["slice_qp"] = qp
    p["tools"] = ((pkg.TOOL_DEP_QUANT if opts & OPT_DQ else 0) | (pkg.TOOL_DEBLOCK if opts & OPT_DBF else 0) |
                  (pkg.TOOL_ENC_FULL_INTRA if opts & OPT_FULL else 0) | (pkg.TOOL_ENC_CCLM if opts & OPT_CCLM else 0))
    p["alf_aps"] = -1
    return p


def _coded_planes(ctx, pkg, pics):
    outs = []
    for p in pics:
        w, h, cf = int(p["width"]), int(p["height"]), int(p["chroma_format"])
        cw, ch = pkg.chroma_dims(w, h, cf)
        outs.append((np.zeros((h, w), np.uint16), np.zeros((ch, cw), np.uint16) if cf else None,
                     np.zeros((ch, cw), np.uint16) if cf else None))
    return outs


def _check_picture(i, p, cus_g, lv_g, rec_g, cus_o, lv_o, rec_o):
    tb = min(1 << int(p["ctu_log2"]), 32)
    cf = int(p["chroma_format"])
    n = [tb * tb] + [len(lv_g)] * 2
    if cf:
        sw = 2 if cf in (1, 2) else 1
        sh = 2 if cf == 1 else 1
        n[1] = n[2] = max(tb // sw, 2) * max(tb // sh, 2)
    for f in ("luma_mode", "chroma_mode", "cbf"):
        bad = np.nonzero(cus_g[f] != cus_o[f])[0]
        assert bad.size == 0, f"picture {i}: {f} differs at CU {bad[:5].tolist()}"
    for k in range(len(cus_o)):
        for c in range(3 if cf else 1):
            if cus_o["cbf"][k] >> c & 1:
                og, oo = int(cus_g["level_off"][k, c]), int(cus_o["level_off"][k, c])
                assert (lv_g[og:og + n[c]] == lv_o[oo:oo + n[c]]).all(), f"picture {i} CU {k} comp {c} levels"
            else:
                assert cus_g["level_off"][k, c] == -1
    for c in range(3 if cf else 1):
        diff = np.argwhere(rec_g[c] != rec_o[c][:rec_g[c].shape[0], :rec_g[c].shape[1]])
        assert diff.size == 0, f"picture {i} plane {c}: {len(diff)} samples differ, first {diff[:3].tolist()}"


@pytest.mark.parametrize("bd,qp,ctu_log2,opts,cf", [
    (10, 22, 5, OPT_FULL | OPT_CCLM | OPT_DBF, 1),
    (10, 37, 5, OPT_FULL | OPT_CCLM | OPT_DQ | OPT_DBF, 1),
    (8, 30, 6, OPT_FULL | OPT_CCLM, 1),
    (12, 27, 7, OPT_FULL | OPT_DBF, 1),
    (10, 32, 5, OPT_DBF, 1),
    (10, 27, 5, OPT_FULL | OPT_CCLM | OPT_DBF, 2),
    (10, 27, 6, OPT_FULL | OPT_CCLM | OPT_DQ, 3),
    (10, 25, 5, OPT_FULL | OPT_DQ | OPT_DBF, 0),
    (10, 4, 5, OPT_FULL | OPT_CCLM, 1),
])
def test_encoder_matches_oracle(ctx, pkg, orc, bd, qp, ctu_log2, opts, cf):
    from rustmpeg_next_b200 import synth

    ctu = 1 << ctu_log2
    w, h = -(-200 // ctu) * ctu, -(-120 // ctu) * ctu
    y, u, v = synth.source_planes(w, h, bd, cf, seed=qp, vis=(200, 120))
    cus_o, lv_o, rec_o = orc.encode_frame(y, u, v, bd, qp, ctu_log2, opts, cf=cf)
    p = _desc(pkg, w, h, bd, qp, ctu_log2, opts, cf)
    cus_g, lv_g = ctx.encode_batch(np.array([p]), [(y, u, v)])
    rec_g = ctx.download(_coded_planes(ctx, pkg, [p]))[0]
    _check_picture(0, p, cus_g, lv_g, rec_g, cus_o, lv_o, rec_o)


def test_encoder_batch_of_mixed_pictures_and_closed_loop(ctx, pkg, orc):
    from rustmpeg_next_b200 import synth

    cfgs = [(256, 128, 10, 27, 5, OPT_FULL | OPT_CCLM | OPT_DBF, 1), (128, 128, 8, 32, 6, OPT_FULL | OPT_DQ, 1),
            (96, 64, 12, 22, 5, OPT_FULL | OPT_CCLM | OPT_DBF, 3), (256, 256, 10, 37, 7, OPT_DBF, 1),
            (64, 96, 10, 30, 5, OPT_FULL | OPT_CCLM | OPT_DQ | OPT_DBF, 2)]
    pics, srcs, want = [], [], []
    for i, (w, h, bd, qp, cl, opts, cf) in enumerate(cfgs):
        y, u, v = synth.source_planes(w, h, bd, cf, seed=100 + i)
        pics.append(_desc(pkg, w, h, bd, qp, cl, opts, cf))
        srcs.append((y, u, v))
        want.append(orc.encode_frame(y, u, v, bd, qp, cl, opts, cf=cf))
    pics = np.array(pics)
    cus_g, lv_g = ctx.encode_batch(pics, srcs)
    recs = ctx.download(_coded_planes(ctx, pkg, pics))
    at = 0
    for i, p in enumerate(pics):
        tb = min(1 << int(p["ctu_log2"]), 32)
        n = (int(p["width"]) // tb) * (int(p["height"]) // tb)
        _check_picture(i, p, cus_g[at:at + n], lv_g, recs[i], *want[i])
        at += n
    # closed loop: decode the emitted records (slice.rs round-trip tests)
    pics["chroma_qp_scaled"] = [orc.chroma_qp(int(p["slice_qp"]), int(p["bit_depth"])) for p in pics]
    pics["cu_offset"] = np.cumsum([0] + [(int(p["width"]) // min(1 << int(p["ctu_log2"]), 32)) *
                                         (int(p["height"]) // min(1 << int(p["ctu_log2"]), 32)) for p in pics])[:-1]
    nctu = sum((int(p["width"]) >> int(p["ctu_log2"])) * (int(p["height"]) >> int(p["ctu_log2"])) for p in pics)
    dec = ctx.decode_batch(pkg.Batch(pics, cus_g, lv_g, np.zeros(nctu, pkg.CTU_DTYPE)), _coded_planes(ctx, pkg, pics))
    for i in range(len(pics)):
        for c in range(3):
            if recs[i][c] is not None:
                assert (dec[i][c] == recs[i][c]).all(), f"closed loop: picture {i} plane {c}"
