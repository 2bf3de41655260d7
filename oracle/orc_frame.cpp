// CPU oracle (test infrastructure only; see oracle.h): the 8..12-bit frame
// path of the reference's subset coder, slice::encode_vvc_frame_picture
// (slice.rs:4171-4634) and slice::decode_vvc_frame_picture_with_chroma_qp
// (slice.rs:4659-5072), restated without the CABAC layer. The encoder emits
// the coding-unit records and transform levels that a CABAC parse of its
// bitstream yields; the decoder reconstructs and filters a picture from
// such records. Both use the record layout of include/vvcg.h.
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "../include/vvcg.h"
#include "oracle.h"

namespace orc {

struct FrameGeom {
  int w, h, bd, cf, ctu, tb, sub_w, sub_h, tb_cw, tb_ch, cw, ch;
};

static bool make_geom(int w, int h, int bd, int cf, int ctu_log2, FrameGeom* g) {
  if (ctu_log2 < 5 || ctu_log2 > 7) return false;  // slice.rs:129-160 validate_coded_geometry
  int ctu = 1 << ctu_log2;
  if (w < ctu || h < ctu || w % ctu || h % ctu) return false;
  if (bd < 8 || bd > 12 || cf < 0 || cf > 3) return false;
  g->w = w;
  g->h = h;
  g->bd = bd;
  g->cf = cf;
  g->ctu = ctu;
  g->tb = std::min(ctu, 32);
  g->sub_w = (cf == 1 || cf == 2) ? 2 : 1;
  g->sub_h = cf == 1 ? 2 : 1;
  bool has_c = cf != 0;
  g->tb_cw = has_c ? std::max(g->tb / g->sub_w, 2) : 0;
  g->tb_ch = has_c ? std::max(g->tb / g->sub_h, 2) : 0;
  g->cw = has_c ? (w + g->sub_w - 1) / g->sub_w : 0;
  g->ch = has_c ? (h + g->sub_h - 1) / g->sub_h : 0;
  return true;
}

// slice.rs:164-187 coding_unit_order
static std::vector<std::pair<int, int>> coding_unit_order(int ctu, int tb, int w, int h) {
  std::vector<std::pair<int, int>> offs{{0, 0}};
  for (int step = ctu / 2; step >= tb; step /= 2) {
    std::vector<std::pair<int, int>> next;
    for (auto& o : offs) {
      next.push_back({o.first, o.second});
      next.push_back({o.first + step, o.second});
      next.push_back({o.first, o.second + step});
      next.push_back({o.first + step, o.second + step});
    }
    offs.swap(next);
  }
  std::vector<std::pair<int, int>> order;
  for (int cy = 0; cy < h; cy += ctu)
    for (int cx = 0; cx < w; cx += ctu)
      for (auto& o : offs) order.push_back({cx + o.first, cy + o.second});
  return order;
}

static void reconstruct_tb(const int16_t* lv, int w, int h, int qp_scaled, int bd, bool dq,
                           int32_t* res) {
  std::vector<int32_t> levels(w * h), d(w * h), scan(w * h);
  for (int i = 0; i < w * h; i++) levels[i] = lv[i];
  if (dq) {
    coeff_scan_raster(w, h, scan.data());
    dequantize_dep_quant_bd(w, h, levels.data(), scan.data(), qp_scaled, bd, d.data());
  } else {
    dequantize_rect_bd(w, h, levels.data(), qp_scaled, bd, d.data());
  }
  inverse_transform_rect_bd(w, h, d.data(), kDct2, kDct2, 0, 0, bd, res);
}

// One encoded TB: forward transform, quantisation and the encoder's own
// reconstruction (slice.rs:4298-4346 for luma, :4442-4553 for chroma).
static bool code_tb(const int32_t* resid, int w, int h, int qp_scaled, int bd, bool dq,
                    int32_t* levels, int32_t* recon_res) {
  std::vector<int32_t> coeff(w * h), scan(w * h), d(w * h);
  forward_transform_rect_bd(w, h, resid, kDct2, kDct2, 0, 0, bd, coeff.data());
  if (dq) {
    coeff_scan_raster(w, h, scan.data());
    quantize_dep_quant_bd(w, h, coeff.data(), scan.data(), qp_scaled, bd, levels);
    dequantize_dep_quant_bd(w, h, levels, scan.data(), qp_scaled, bd, d.data());
  } else {
    quantize_rect_bd(w, h, coeff.data(), qp_scaled, bd, true, levels);
    dequantize_rect_bd(w, h, levels, qp_scaled, bd, d.data());
  }
  inverse_transform_rect_bd(w, h, d.data(), kDct2, kDct2, 0, 0, bd, recon_res);
  for (int i = 0; i < w * h; i++)
    if (levels[i] != 0) return true;
  return false;
}

struct LevelSink {
  int16_t* pool;
  uint64_t cap;
  uint64_t used;
  int32_t push(const int32_t* lv, int n) {
    if (used + n > cap) return -2;
    int32_t off = (int32_t)used;
    for (int i = 0; i < n; i++) pool[used + i] = (int16_t)lv[i];
    used += n;
    return off;
  }
};

static void deblock_picture(Plane16& y, Plane16& u, Plane16& v, const FrameGeom& g, int qp) {
  // slice.rs:4993-5020 (decoder) / :4603-4630 (encoder)
  deblock_luma_plane_16(y, g.tb, g.ctu, qp, 2, 0, 0);
  if (g.cf != 0) {
    int c_qp = std::min(63, std::max(0, derived_chroma_qp(qp)));
    deblock_chroma_plane_16(u, g.tb_cw, g.ctu / g.sub_h, c_qp, 2, 0, 0, g.sub_w, g.sub_h);
    deblock_chroma_plane_16(v, g.tb_cw, g.ctu / g.sub_h, c_qp, 2, 0, 0, g.sub_w, g.sub_h);
  }
}

}  // namespace orc

using namespace orc;

extern "C" {

// Options of orc_encode_frame (SliceCodingOptions, slice.rs:1472-1510).
enum {
  ORC_OPT_FULL_INTRA = 1,
  ORC_OPT_CCLM = 2,
  ORC_OPT_DEP_QUANT = 4,
  ORC_OPT_DEBLOCK = 8,
};

// slice::encode_vvc_frame_picture (slice.rs:4171-4634) without the CABAC
// writes. src_* are the padded (coded-size) planes. Writes one record per
// tb-grid cell (raster order) and appends the levels of every TB with a
// nonzero level to `levels` in coding order. Returns 0 on success.
int orc_encode_frame(const uint16_t* src_y, const uint16_t* src_u, const uint16_t* src_v, int w,
                     int h, int bd, int cf, int qp, int ctu_log2, int opts, vvcg_cu_rec* cus,
                     int16_t* levels, uint64_t levels_cap, uint64_t* levels_used, uint16_t* rec_y,
                     uint16_t* rec_u, uint16_t* rec_v) {
  FrameGeom g;
  if (!make_geom(w, h, bd, cf, ctu_log2, &g)) return -1;
  bool has_c = cf != 0;
  int lqp = std::max(scaled_luma_qp_bd(qp, bd), 4);
  int cqp = std::max(derived_chroma_qp_bd(qp, bd, 0), 4);
  bool dq = opts & ORC_OPT_DEP_QUANT;
  int maxv = (1 << bd) - 1;
  memset(rec_y, 0, sizeof(uint16_t) * w * h);
  if (has_c) {
    memset(rec_u, 0, sizeof(uint16_t) * g.cw * g.ch);
    memset(rec_v, 0, sizeof(uint16_t) * g.cw * g.ch);
  }
  Plane16 sy{(uint16_t*)src_y, w, h, bd}, su{(uint16_t*)src_u, g.cw, g.ch, bd},
      sv{(uint16_t*)src_v, g.cw, g.ch, bd};
  Plane16 ry{rec_y, w, h, bd}, ru{rec_u, g.cw, g.ch, bd}, rv{rec_v, g.cw, g.ch, bd};
  int gw = w / g.tb, gh = h / g.tb;
  std::vector<uint8_t> coded(gw * gh, 0);
  CodedMap cm{coded.data(), gw, gh, g.tb};
  LevelSink sink{levels, levels_cap, 0};
  int tb = g.tb, tcw = g.tb_cw, tch = g.tb_ch;
  std::vector<uint16_t> pred(tb * tb), pu(tcw * tch + 1), pv(tcw * tch + 1), ptmp(tcw * tch + 1);
  std::vector<int32_t> res(tb * tb), lv(tb * tb), rr(tb * tb);
  std::vector<int32_t> resu(tcw * tch + 1), resv(tcw * tch + 1), lvu(tcw * tch + 1),
      lvv(tcw * tch + 1), rru(tcw * tch + 1), rrv(tcw * tch + 1);
  for (auto& pos : coding_unit_order(g.ctu, tb, w, h)) {
    int bx = pos.first, by = pos.second;
    int gx = bx / tb, gy = by / tb;
    int cx = bx / g.sub_w, cy = by / g.sub_h;
    coded[gy * gw + gx] = 1;
    vvcg_cu_rec& rec = cus[gy * gw + gx];
    memset(&rec, 0, sizeof(rec));
    rec.level_off[0] = rec.level_off[1] = rec.level_off[2] = -1;
    // slice.rs:4264-4274 luma mode decision (7-mode SAD; restricted to Planar/DC)
    int m = choose_intra_mode_16(ry, sy, bx, by, tb, tb, true);
    int luma_mode = (opts & ORC_OPT_FULL_INTRA) ? m : ((m == 0 || m == 1) ? m : 0);
    rec.luma_mode = (uint8_t)luma_mode;
    predict_coded_block_16(ry, bx, by, tb, tb, true, luma_mode, 1, 1, cm, pred.data());
    for (int y = 0; y < tb; y++)
      for (int x = 0; x < tb; x++)
        res[y * tb + x] = (int)sy.get(bx + x, by + y) - (int)pred[y * tb + x];
    bool cbf_y = code_tb(res.data(), tb, tb, lqp, bd, dq, lv.data(), rr.data());
    for (int y = 0; y < tb; y++)
      for (int x = 0; x < tb; x++)
        ry.set(bx + x, by + y, std::min(maxv, std::max(0, (int)pred[y * tb + x] + rr[y * tb + x])));
    if (cbf_y) {
      rec.level_off[0] = sink.push(lv.data(), tb * tb);
      if (rec.level_off[0] < 0) return -2;
    }
    int chroma_mode = luma_mode;
    bool cbf_u = false, cbf_v = false;
    if (has_c) {
      if (opts & ORC_OPT_CCLM) {  // slice.rs:4362-4397 chroma mode by SAD
        predict_block_16(ru, cx, cy, tcw, tch, false, luma_mode, ptmp.data());
        uint64_t best = 0;
        for (int y = 0; y < tch; y++)
          for (int x = 0; x < tcw; x++)
            best += (uint64_t)std::abs((int)su.get(cx + x, cy + y) - (int)ptmp[y * tcw + x]);
        for (int k = 0; k < 3; k++) {
          predict_cclm_with_format_16(ry, ru, cx, cy, tcw, tch, k, cf, g.ctu, ptmp.data());
          uint64_t sad = 0;
          for (int y = 0; y < tch; y++)
            for (int x = 0; x < tcw; x++)
              sad += (uint64_t)std::abs((int)su.get(cx + x, cy + y) - (int)ptmp[y * tcw + x]);
          if (sad < best) {
            best = sad;
            chroma_mode = 81 + k;
          }
        }
      }
      if (chroma_mode >= 81 && chroma_mode <= 83) {
        predict_cclm_with_format_16(ry, ru, cx, cy, tcw, tch, chroma_mode - 81, cf, g.ctu, pu.data());
        predict_cclm_with_format_16(ry, rv, cx, cy, tcw, tch, chroma_mode - 81, cf, g.ctu, pv.data());
      } else {
        int cm_mode = chroma_mode <= 69 ? chroma_mode : 0;  // slice.rs:1980 ipm
        predict_coded_block_16(ru, cx, cy, tcw, tch, false, cm_mode, g.sub_w, g.sub_h, cm, pu.data());
        predict_coded_block_16(rv, cx, cy, tcw, tch, false, cm_mode, g.sub_w, g.sub_h, cm, pv.data());
      }
      for (int y = 0; y < tch; y++)
        for (int x = 0; x < tcw; x++) {
          resu[y * tcw + x] = (int)su.get(cx + x, cy + y) - (int)pu[y * tcw + x];
          resv[y * tcw + x] = (int)sv.get(cx + x, cy + y) - (int)pv[y * tcw + x];
        }
      cbf_u = code_tb(resu.data(), tcw, tch, cqp, bd, dq, lvu.data(), rru.data());
      cbf_v = code_tb(resv.data(), tcw, tch, cqp, bd, dq, lvv.data(), rrv.data());
      for (int y = 0; y < tch; y++)
        for (int x = 0; x < tcw; x++) {
          ru.set(cx + x, cy + y, std::min(maxv, std::max(0, (int)pu[y * tcw + x] + rru[y * tcw + x])));
          rv.set(cx + x, cy + y, std::min(maxv, std::max(0, (int)pv[y * tcw + x] + rrv[y * tcw + x])));
        }
      if (cbf_u) {
        rec.level_off[1] = sink.push(lvu.data(), tcw * tch);
        if (rec.level_off[1] < 0) return -2;
      }
      if (cbf_v) {
        rec.level_off[2] = sink.push(lvv.data(), tcw * tch);
        if (rec.level_off[2] < 0) return -2;
      }
    }
    rec.chroma_mode = (uint8_t)chroma_mode;
    rec.cbf = (uint8_t)((cbf_y ? 1 : 0) | (cbf_u ? 2 : 0) | (cbf_v ? 4 : 0));
  }
  if (opts & ORC_OPT_DEBLOCK) deblock_picture(ry, ru, rv, g, qp);
  *levels_used = sink.used;
  return 0;
}

// Reconstruction and loop filters of slice::decode_vvc_frame_picture_with_chroma_qp
// (slice.rs:4834-5072) for one picture, from its records. `cus` and `ctus` point
// at the picture's first record; level offsets index `levels`. Output planes
// have the coded size. Returns 0, or -3 when the reference would abort
// (fixed-filter ALF reaching a class >= 16, filter.rs:2072).
int orc_recon_frame(const vvcg_pic_desc* pic, const vvcg_cu_rec* cus, const int16_t* levels,
                    const vvcg_ctu_filter* ctus, const vvcg_alf_aps* aps, uint16_t* out_y,
                    uint16_t* out_u, uint16_t* out_v) {
  FrameGeom g;
  if (!make_geom((int)pic->width, (int)pic->height, pic->bit_depth, pic->chroma_format,
                 pic->ctu_log2, &g))
    return -1;
  int w = g.w, h = g.h, bd = g.bd, cf = g.cf;
  bool has_c = cf != 0;
  int qp = pic->slice_qp;
  int lqp = std::max(scaled_luma_qp_bd(qp, bd), 4);
  int cqp = std::max((int)pic->chroma_qp_scaled, 4);
  bool dq = pic->tools & VVCG_TOOL_DEP_QUANT;
  int maxv = (1 << bd) - 1;
  memset(out_y, 0, sizeof(uint16_t) * w * h);
  if (has_c) {
    memset(out_u, 0, sizeof(uint16_t) * g.cw * g.ch);
    memset(out_v, 0, sizeof(uint16_t) * g.cw * g.ch);
  }
  Plane16 ry{out_y, w, h, bd}, ru{out_u, g.cw, g.ch, bd}, rv{out_v, g.cw, g.ch, bd};
  int gw = w / g.tb, gh = h / g.tb;
  std::vector<uint8_t> coded(gw * gh, 0);
  CodedMap cm{coded.data(), gw, gh, g.tb};
  int tb = g.tb, tcw = g.tb_cw, tch = g.tb_ch;
  std::vector<uint16_t> pred(tb * tb), pu(tcw * tch + 1), pv(tcw * tch + 1);
  std::vector<int32_t> rr(tb * tb), rru(tcw * tch + 1), rrv(tcw * tch + 1);
  for (auto& pos : coding_unit_order(g.ctu, tb, w, h)) {
    int bx = pos.first, by = pos.second;
    int gx = bx / tb, gy = by / tb;
    int cx = bx / g.sub_w, cy = by / g.sub_h;
    coded[gy * gw + gx] = 1;
    const vvcg_cu_rec& rec = cus[gy * gw + gx];
    int lm = rec.luma_mode <= 69 ? rec.luma_mode : 0;
    predict_coded_block_16(ry, bx, by, tb, tb, true, lm, 1, 1, cm, pred.data());
    if ((rec.cbf & 1) && rec.level_off[0] >= 0)
      reconstruct_tb(levels + rec.level_off[0], tb, tb, lqp, bd, dq, rr.data());
    else
      std::fill(rr.begin(), rr.end(), 0);
    for (int y = 0; y < tb; y++)
      for (int x = 0; x < tb; x++)
        ry.set(bx + x, by + y, std::min(maxv, std::max(0, (int)pred[y * tb + x] + rr[y * tb + x])));
    if (!has_c) continue;
    int chm = rec.chroma_mode;
    if (chm >= 81 && chm <= 83) {
      predict_cclm_with_format_16(ry, ru, cx, cy, tcw, tch, chm - 81, cf, g.ctu, pu.data());
      predict_cclm_with_format_16(ry, rv, cx, cy, tcw, tch, chm - 81, cf, g.ctu, pv.data());
    } else {
      int cmode = chm <= 69 ? chm : 0;
      predict_coded_block_16(ru, cx, cy, tcw, tch, false, cmode, g.sub_w, g.sub_h, cm, pu.data());
      predict_coded_block_16(rv, cx, cy, tcw, tch, false, cmode, g.sub_w, g.sub_h, cm, pv.data());
    }
    if ((rec.cbf & 2) && rec.level_off[1] >= 0)
      reconstruct_tb(levels + rec.level_off[1], tcw, tch, cqp, bd, dq, rru.data());
    else
      std::fill(rru.begin(), rru.end(), 0);
    if ((rec.cbf & 4) && rec.level_off[2] >= 0)
      reconstruct_tb(levels + rec.level_off[2], tcw, tch, cqp, bd, dq, rrv.data());
    else
      std::fill(rrv.begin(), rrv.end(), 0);
    for (int y = 0; y < tch; y++)
      for (int x = 0; x < tcw; x++) {
        ru.set(cx + x, cy + y, std::min(maxv, std::max(0, (int)pu[y * tcw + x] + rru[y * tcw + x])));
        rv.set(cx + x, cy + y, std::min(maxv, std::max(0, (int)pv[y * tcw + x] + rrv[y * tcw + x])));
      }
  }
  if (pic->tools & VVCG_TOOL_DEBLOCK) deblock_picture(ry, ru, rv, g, qp);
  int cgw = w / g.ctu, cgh = h / g.ctu;
  if (pic->tools & VVCG_TOOL_SAO) {  // slice.rs:5022-5054
    std::vector<uint16_t> cy_(out_y, out_y + (size_t)w * h);
    std::vector<uint16_t> cu_(has_c ? (size_t)g.cw * g.ch : 1), cv_(has_c ? (size_t)g.cw * g.ch : 1);
    if (has_c) {
      memcpy(cu_.data(), out_u, sizeof(uint16_t) * g.cw * g.ch);
      memcpy(cv_.data(), out_v, sizeof(uint16_t) * g.cw * g.ch);
    }
    Plane16 sy{cy_.data(), w, h, bd}, su{cu_.data(), g.cw, g.ch, bd}, sv{cv_.data(), g.cw, g.ch, bd};
    int ctu_cw = has_c ? g.ctu / g.sub_w : 0, ctu_ch = has_c ? g.ctu / g.sub_h : 0;
    for (int yy = 0; yy < cgh; yy++)
      for (int xx = 0; xx < cgw; xx++) {
        const vvcg_ctu_filter& f = ctus[yy * cgw + xx];
        Sao s[3];
        for (int c = 0; c < 3; c++) {
          s[c].type = f.sao[c].type;
          s[c].band_pos_or_class = f.sao[c].band_or_class;
          for (int k = 0; k < 4; k++) s[c].offsets[k] = f.sao[c].offsets[k];
        }
        if (apply_sao_region_16(sy, ry, xx * g.ctu, yy * g.ctu, g.ctu, g.ctu, s[0])) return -3;
        if (has_c) {
          if (apply_sao_region_16(su, ru, xx * ctu_cw, yy * ctu_ch, ctu_cw, ctu_ch, s[1])) return -3;
          if (apply_sao_region_16(sv, rv, xx * ctu_cw, yy * ctu_ch, ctu_cw, ctu_ch, s[2])) return -3;
        }
      }
  }
  if (pic->tools & VVCG_TOOL_ALF) {  // slice.rs:5055-5069: any CTU flag -> whole luma plane
    bool any = false;
    for (int i = 0; i < cgw * cgh; i++) any |= ctus[i].alf_luma != 0;
    if (any) {
      AlfAps a;
      memset(&a, 0, sizeof(a));
      if (aps) {
        a.num_luma_filters = aps->num_luma_filters;
        a.luma_clip = aps->luma_clip;
        memcpy(a.coeff_delta_idx, aps->coeff_delta_idx, 25);
        memcpy(a.coeff, aps->coeff, sizeof(a.coeff));
        memcpy(a.clip_idx, aps->clip_idx, sizeof(a.clip_idx));
      }
      apply_alf_luma_plane_16(ry, a);
      if (orc::g_alf_status != 0) return -3;
    }
  }
  return 0;
}

}  // extern "C"
