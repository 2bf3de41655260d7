// CPU oracle (test infrastructure only; see oracle.h): flat extern "C" entry
// points over the restated reference functions, for the Python tests and the
// CPU legs of bench.py (loaded with ctypes). Each wraps one function of the
// oracle with plain pointers; planes are row-major with stride = width.
#include <string.h>

#include <vector>

#include "oracle.h"

using namespace orc;

extern "C" {

int orc_forward_transform(int w, int h, const int32_t* res, int trh, int trv, int esw, int esh,
                          int bd, int32_t* out) {
  return forward_transform_rect_bd(w, h, res, trh, trv, esw, esh, bd, out);
}
int orc_inverse_transform(int w, int h, const int32_t* co, int trh, int trv, int esw, int esh,
                          int bd, int32_t* out) {
  return inverse_transform_rect_bd(w, h, co, trh, trv, esw, esh, bd, out);
}
int orc_quantize(int w, int h, const int32_t* c, int qp, int bd, int intra, int32_t* out) {
  return quantize_rect_bd(w, h, c, qp, bd, intra != 0, out);
}
int orc_dequantize(int w, int h, const int32_t* l, int qp, int bd, int32_t* out) {
  return dequantize_rect_bd(w, h, l, qp, bd, out);
}
int orc_quantize_dq(int w, int h, const int32_t* c, int qp, int bd, int32_t* out) {
  std::vector<int32_t> scan(w * h);
  coeff_scan_raster(w, h, scan.data());
  return quantize_dep_quant_bd(w, h, c, scan.data(), qp, bd, out);
}
int orc_dequantize_dq(int w, int h, const int32_t* l, int qp, int bd, int32_t* out) {
  std::vector<int32_t> scan(w * h);
  coeff_scan_raster(w, h, scan.data());
  return dequantize_dep_quant_bd(w, h, l, scan.data(), qp, bd, out);
}
int orc_coeff_scan(int w, int h, int32_t* raster) { return coeff_scan_raster(w, h, raster); }
int orc_quantize_ts(int r, int qp) { return quantize_ts(r, qp); }
int orc_dequantize_ts(int l, int qp) { return dequantize_ts(l, qp); }
int orc_scaled_luma_qp(int qp, int bd) { return scaled_luma_qp_bd(qp, bd); }
int orc_chroma_qp(int qp, int bd, int off) { return derived_chroma_qp_bd(qp, bd, off); }
int orc_wide_angle(int w, int h, int mode) { return get_modified_wide_angle(w, h, mode); }
void orc_angular_params(int mode, int w, int h, int is_luma, int32_t* out8) {
  AngularParams p = init_angular_params(mode, w, h, w, h, is_luma != 0, 0, false);
  out8[0] = p.pred_mode;
  out8[1] = p.is_mode_ver;
  out8[2] = p.intra_pred_angle;
  out8[3] = p.abs_inv_angle;
  out8[4] = p.ref_filter_flag;
  out8[5] = p.interpolation_flag;
  out8[6] = p.apply_pdpc;
  out8[7] = p.angular_scale;
}

void orc_predict_block(const uint16_t* plane, int pw, int ph, int bd, int x, int y, int w, int h,
                       int is_luma, int mode, uint16_t* out) {
  Plane16 p{(uint16_t*)plane, pw, ph, bd};
  predict_block_16(p, x, y, w, h, is_luma != 0, mode, out);
}
// `coded` is the tb-grid availability map of predict_coded_block_16.
void orc_predict_coded_block(const uint16_t* plane, int pw, int ph, int bd, int x, int y, int w,
                             int h, int is_luma, int mode, int sx, int sy, const uint8_t* coded,
                             int gw, int gh, int tb, uint16_t* out) {
  Plane16 p{(uint16_t*)plane, pw, ph, bd};
  CodedMap cm{coded, gw, gh, tb};
  predict_coded_block_16(p, x, y, w, h, is_luma != 0, mode, sx, sy, cm, out);
}
void orc_predict_cclm(const uint16_t* luma, int lw, int lh, const uint16_t* chroma, int cw_, int ch_,
                      int bd, int bxc, int byc, int cw, int ch, int mode, int cf, int ctu,
                      uint16_t* out) {
  Plane16 l{(uint16_t*)luma, lw, lh, bd}, c{(uint16_t*)chroma, cw_, ch_, bd};
  predict_cclm_with_format_16(l, c, bxc, byc, cw, ch, mode, cf, ctu, out);
}
int orc_choose_intra_mode(const uint16_t* recon, const uint16_t* src, int pw, int ph, int bd,
                          int bx, int by, int w, int h) {
  Plane16 r{(uint16_t*)recon, pw, ph, bd}, s{(uint16_t*)src, pw, ph, bd};
  return choose_intra_mode_16(r, s, bx, by, w, h, true);
}

void orc_deblock_luma(uint16_t* plane, int pw, int ph, int bd, int cu_step, int ctb, int qp, int bs,
                      int beta_off, int tc_off) {
  Plane16 p{plane, pw, ph, bd};
  deblock_luma_plane_16(p, cu_step, ctb, qp, bs, beta_off, tc_off);
}
void orc_deblock_chroma(uint16_t* plane, int pw, int ph, int bd, int cu_step, int ctb_h, int qp,
                        int bs, int beta_off, int tc_off, int sub_w, int sub_h) {
  Plane16 p{plane, pw, ph, bd};
  deblock_chroma_plane_16(p, cu_step, ctb_h, qp, bs, beta_off, tc_off, sub_w, sub_h);
}
int orc_sao_region(const uint16_t* src, uint16_t* dst, int pw, int ph, int bd, int bx, int by,
                   int w, int h, int type, int band_or_class, const int32_t* offsets) {
  Plane16 s{(uint16_t*)src, pw, ph, bd}, d{dst, pw, ph, bd};
  Sao sao{type, band_or_class, {offsets[0], offsets[1], offsets[2], offsets[3]}};
  return apply_sao_region_16(s, d, bx, by, w, h, sao);
}
// aps == NULL selects the fixed filters. Returns -1 where the reference aborts.
int orc_alf_luma(uint16_t* plane, int pw, int ph, int bd, int num_filters, int luma_clip,
                 const uint8_t* delta_idx, const int16_t* coeff, const uint8_t* clip_idx) {
  Plane16 p{plane, pw, ph, bd};
  AlfAps a;
  memset(&a, 0, sizeof(a));
  a.num_luma_filters = num_filters;
  a.luma_clip = luma_clip != 0;
  if (num_filters > 0) {
    memcpy(a.coeff_delta_idx, delta_idx, 25);
    memcpy(a.coeff, coeff, sizeof(int16_t) * 25 * 12);
    memcpy(a.clip_idx, clip_idx, 25 * 12);
  }
  apply_alf_luma_plane_16(p, a);
  return g_alf_status;
}
void orc_alf_classify(const uint16_t* plane, int pw, int ph, int bd, int bx, int by,
                      int32_t* out2) {
  Plane16 p{(uint16_t*)plane, pw, ph, bd};
  classify_alf_4x4_16(p, bx, by, &out2[0], &out2[1]);
}

void orc_mc_luma(const uint16_t* ref, int pw, int ph, int bd, int bx, int by, int w, int h, int mvx,
                 int mvy, int bi, int affine, int alt_hpel, int32_t* out) {
  Plane16 p{(uint16_t*)ref, pw, ph, bd};
  interpolate_luma_block_16(p, bx, by, w, h, mvx, mvy, bi != 0, affine != 0, alt_hpel != 0, out);
}
void orc_mc_chroma(const uint16_t* ref, int pw, int ph, int bd, int bxc, int byc, int cw, int ch,
                   int mvx, int mvy, int bi, int cf, int32_t* out) {
  Plane16 p{(uint16_t*)ref, pw, ph, bd};
  interpolate_chroma_block_format_16(p, bxc, byc, cw, ch, mvx, mvy, bi != 0, cf, out);
}
void orc_bi_average(const int32_t* p0, const int32_t* p1, int n, int bcw, int bd, uint16_t* out) {
  weighted_average_bi_16(p0, p1, n, bcw, bd, out);
}

// Runs every record of a transform-unit batch; returns 0, or -(i + 1) for
// the first record the reference rejects.
int orc_tu_batch(int forward, const void* recs, int n, const int16_t* in, int16_t* out) {
  const TuRec* r = (const TuRec*)recs;
  for (int i = 0; i < n; i++) {
    int rc = forward ? tu_forward(r[i], in + r[i].in_off, out + r[i].out_off)
                     : tu_inverse(r[i], in + r[i].in_off, out + r[i].out_off);
    if (rc) return -(i + 1);
  }
  return 0;
}

}  // extern "C"

// crates/rustmpeg-video/src/accelerator.rs:258-292 CpuFrameMetrics::plane_metrics
// over `elem`-byte samples (1 or 2), strides in samples; out = {sse, sad, samples}.
extern "C" int orc_plane_metrics(const void* a, uint64_t sa, const void* b, uint64_t sb, uint32_t w,
                                 uint32_t h, int elem, uint64_t* out) {
  out[0] = out[1] = out[2] = 0;
  if (w == 0 || h == 0) return 0;
  if (sa < w || sb < w) return -1;
  uint64_t sse = 0, sad = 0;
  for (uint32_t y = 0; y < h; y++)
    for (uint32_t x = 0; x < w; x++) {
      int l = elem == 1 ? ((const uint8_t*)a)[y * sa + x] : ((const uint16_t*)a)[y * sa + x];
      int r = elem == 1 ? ((const uint8_t*)b)[y * sb + x] : ((const uint16_t*)b)[y * sb + x];
      uint64_t d = (uint64_t)(l > r ? l - r : r - l);
      sse += d * d;
      sad += d;
    }
  out[0] = sse;
  out[1] = sad;
  out[2] = (uint64_t)w * h;
  return 0;
}

extern "C" void orc_mc_luma_8(const uint8_t* ref, int pw, int ph, int stride, int bx, int by, int w, int h,
                              int mvx, int mvy, int bi, int alt_hpel, int affine, int32_t* out) {
  orc::interpolate_luma_block_8(ref, pw, ph, stride, bx, by, w, h, mvx, mvy, bi, alt_hpel, affine, out);
}
extern "C" void orc_mc_chroma_420_8(const uint8_t* ref, int pw, int ph, int stride, int cx, int cy, int cw,
                                    int ch, int mvx, int mvy, int bi, int32_t* out) {
  orc::interpolate_chroma_block_420_8(ref, pw, ph, stride, cx, cy, cw, ch, mvx, mvy, bi, out);
}
extern "C" void orc_bi_average_8(const int32_t* p0, const int32_t* p1, int n, int bcw, int32_t* out) {
  orc::weighted_average_bi_8(p0, p1, n, bcw, out);
}

// out[0..9]: cost, split_cost[6], split, cu_mode, modes packed 4 x 8 bits
extern "C" void orc_ctu_search(const uint16_t* src, int pw, int ph, int bd, int cx, int cy, int split_mask,
                               int n_cand, const uint8_t* cand, uint32_t lambda_q8, uint32_t* out) {
  orc::Plane16 p{(uint16_t*)src, pw, ph, bd};
  int split, cu_mode, modes[4];
  orc::ctu_search(p, cx, cy, split_mask, n_cand, cand, lambda_q8, &out[0], &out[1], &split, &cu_mode, modes);
  out[7] = (uint32_t)split;
  out[8] = (uint32_t)cu_mode;
  out[9] = (uint32_t)(modes[0] | (modes[1] << 8) | (modes[2] << 16) | ((uint32_t)modes[3] << 24));
}
// lfnst.rs forward_lfnst_rect / inverse_lfnst_rect on a w x h raster block in
// place; returns 0, or non-zero where the reference returns an error
extern "C" int orc_lfnst(int forward, int32_t* coeffs, int w, int h, int idx, int mode) {
  return forward ? orc::forward_lfnst_rect(coeffs, w, h, idx, mode) : orc::inverse_lfnst_rect(coeffs, w, h, idx, mode);
}
// 8-bit planes of pw x ph (row-major): src, then n0 + n1 references back to
// back (L0 first); cands / reqs / out in the vvcg_mv_cand / vvcg_me_req /
// vvcg_me_res layouts
extern "C" void orc_inter_search_8(const uint8_t* src, int pw, int ph, const uint8_t* refs, int n0, int n1,
                                   const vvcg_mv_cand* cands, const vvcg_me_req* reqs, int n, vvcg_me_res* out) {
  std::vector<const uint8_t*> l0, l1;
  for (int i = 0; i < n0; i++) l0.push_back(refs + (size_t)i * pw * ph);
  for (int i = 0; i < n1; i++) l1.push_back(refs + (size_t)(n0 + i) * pw * ph);
  for (int i = 0; i < n; i++) {
    const vvcg_me_req& q = reqs[i];
    orc::estimate_inter_block_8(src, l0.data(), n0, l1.data(), n1, pw, ph, pw, cands + q.cand_off, q.num_cands,
                                q.amvp[0], q.amvp[1], (int)q.x, (int)q.y, q.w, q.h, q.search_range, &out[i]);
  }
}
// regions as (x, y, w, h, qp, min_cb) int64 sextuples; out one split per region
extern "C" void orc_qt_mtt_split(const uint16_t* src, int pw, int ph, int bd, const int64_t* regions, int n,
                                 uint8_t* out) {
  orc::Plane16 p{(uint16_t*)src, pw, ph, bd};
  for (int i = 0; i < n; i++) {
    const int64_t* r = regions + 6 * i;
    out[i] = (uint8_t)orc::qt_mtt_split(p, r[0], r[1], r[2], r[3], (int)r[4], r[5]);
  }
}
// planes Y / Cb / Cr row-major at the given strides; dec_y / dec_c byte maps;
// reqs in the vvcg_gen_intra_req layout; out int16
extern "C" void orc_gen_intra_predict(const uint16_t* y, const uint16_t* u, const uint16_t* v, int sy, int sc,
                                      int width, int height, const uint8_t* dec_y, const uint8_t* dec_c, int bd,
                                      int vert_collocated, int ctu, const vvcg_gen_intra_req* reqs, int n,
                                      int16_t* out) {
  vvcg_gen_intra_state st{};
  st.plane[0] = y;
  st.plane[1] = u;
  st.plane[2] = v;
  st.stride[0] = sy;
  st.stride[1] = st.stride[2] = sc;
  st.width = width;
  st.height = height;
  st.dec_y = dec_y;
  st.dec_c = dec_c;
  st.bit_depth = (uint8_t)bd;
  st.vert_collocated = (uint8_t)vert_collocated;
  st.ctu_size = ctu;
  for (int i = 0; i < n; i++) orc::gen_intra_predict(st, reqs[i], out + reqs[i].out_off);
}
// out: mode, mrl index, SAD (low 32 bits), SAD (high 32 bits)
extern "C" void orc_luma_intra_search_8(const uint8_t* recon, const uint8_t* src, int pw, int ph, int bx, int by,
                                        int w, int h, const uint8_t* mpm, int mpm_only, int mrl, int ctu,
                                        uint32_t* out) {
  orc::Plane8 r{recon, pw, ph}, s{src, pw, ph};
  int mode, mi;
  uint64_t sad;
  orc::luma_intra_search_8(r, s, bx, by, w, h, mpm, mpm_only != 0, mrl != 0, ctu, &mode, &mi, &sad);
  out[0] = (uint32_t)mode;
  out[1] = (uint32_t)mi;
  out[2] = (uint32_t)sad;
  out[3] = (uint32_t)(sad >> 32);
}
extern "C" void orc_predict_luma_8(const uint8_t* recon, int pw, int ph, int bx, int by, int w, int h, int mode,
                                   int mrl, int ctu, int32_t* out) {
  orc::Plane8 r{recon, pw, ph};
  orc::predict_luma_8(r, bx, by, w, h, mode, mrl, ctu, out);
}
// planes row-major with strides (samples); cells / ccells / params in the
// vvcg_dbk_cell / vvcg_dbk_ccell / vvcg_dbk_params layouts
extern "C" void orc_inter_ctu_deblock(uint16_t* y, uint16_t* u, uint16_t* v, int sy, int sc, int w, int h, int ctu,
                                      int qp, const vvcg_ctu_motion* cells) {
  uint16_t* const planes[3] = {y, u, v};
  const int stride[3] = {sy, sc, sc};
  orc::inter_ctu_deblock(planes, stride, w, h, ctu, qp, cells);
}

extern "C" void orc_deblock_general(uint16_t* y, uint16_t* u, uint16_t* v, int sy, int sc, int vis_w, int vis_h,
                                    int bd, int ctu, const vvcg_dbk_cell* cells, int cols, int rows,
                                    const vvcg_dbk_ccell* cc, int ccols, int crows, const vvcg_dbk_params* prm) {
  uint16_t* const planes[3] = {y, u, v};
  const int stride[3] = {sy, sc, sc};
  orc::deblock_general(planes, stride, vis_w, vis_h, bd, ctu, cells, cols, rows, cc, ccols, crows, *prm);
}
extern "C" void orc_dbk_lens(int luma, int size_p, int size_q, int ctb_boundary, int* out) {
  if (luma)
    orc::dbk_luma_lens(size_p, size_q, &out[0], &out[1]);
  else
    orc::dbk_chroma_lens(size_p, size_q, ctb_boundary != 0, &out[0], &out[1]);
}
extern "C" int orc_dbk_bs(int p_intra, int q_intra, int p_cbf, int q_cbf, int tu_edge, int pmv_h, int pmv_v,
                          int qmv_h, int qmv_v, int pref, int qref) {
  return orc::dbk_boundary_strength(p_intra, q_intra, p_cbf, q_cbf, tu_edge, pmv_h, pmv_v, qmv_h, qmv_v, pref, qref);
}
// params: 6 bytes per CTU (type, band_or_class, offsets[4]) as vvcg_sao
extern "C" void orc_sao_bounded(const uint16_t* src, uint16_t* dst, int pw, int ph, int vis_w, int vis_h, int bd,
                                int ctu, int ctu_cols, const uint8_t* params, int n_params) {
  std::vector<orc::Sao> s(n_params);
  for (int i = 0; i < n_params; i++) {
    s[i].type = params[6 * i];
    s[i].band_pos_or_class = params[6 * i + 1];
    for (int k = 0; k < 4; k++) s[i].offsets[k] = (int8_t)params[6 * i + 2 + k];
  }
  orc::sao_plane_bounded_16(src, dst, pw, pw, ph, vis_w, vis_h, bd, ctu, ctu_cols, s.data());
}

// slice.rs:325-455 / :458-627: the strict 8-bit profile's encoder decisions and decoder.
extern "C" int orc_strict_encode(const uint8_t* y, const uint8_t* u, const uint8_t* v, int w, int h, int qp,
                                 int ctu_log2, void* cus, int16_t* levels, uint64_t* num_levels, uint8_t* ry,
                                 uint8_t* ru, uint8_t* rv) {
  return orc::strict_encode(y, u, v, w, h, qp, ctu_log2, (vvcg_cu_rec*)cus, levels, num_levels, ry, ru, rv);
}
extern "C" int orc_strict_decode(const void* cus, const int16_t* levels, uint64_t num_levels, int w, int h, int qp,
                                 int ctu_log2, uint8_t* ry, uint8_t* ru, uint8_t* rv) {
  return orc::strict_decode((const vvcg_cu_rec*)cus, levels, num_levels, w, h, qp, ctu_log2, ry, ru, rv);
}

// cabac.rs / residual.rs / slice.rs encoder side (orc_cabac.cpp): a strict
// picture's slice data, or one residual block's substream. Returns 0 and the
// byte count in *size, -1000 when `cap` is too small, or the writer's code.
extern "C" int orc_strict_write(const void* cus, const int16_t* levels, uint64_t num_levels, int w, int h, int qp,
                                uint8_t* out, uint64_t cap, uint64_t* size) {
  std::vector<uint8_t> b;
  const int rc = orc::strict_write((const vvcg_cu_rec*)cus, levels, num_levels, w, h, qp, &b);
  if (rc) return rc;
  if (b.size() > cap) return -1000;
  memcpy(out, b.data(), b.size());
  *size = b.size();
  return 0;
}
extern "C" int orc_block_write(const int32_t* c, int w, int h, int luma, int dq, int sdh, int ts, int qp, uint8_t* out,
                               uint64_t cap, uint64_t* size) {
  std::vector<uint8_t> b;
  const int rc = orc::block_write(c, w, h, luma != 0, dq != 0, sdh != 0, ts != 0, qp, &b);
  if (rc) return rc;
  if (b.size() > cap) return -1000;
  memcpy(out, b.data(), b.size());
  *size = b.size();
  return 0;
}


// The multi-tool stream (orc_multitool.cpp, orc_cabac.cpp). refs: 3 * num_refs
// plane pointers (Y, Cb, Cr of each L0 picture).
extern "C" int orc_mt_encode(const uint8_t* y, const uint8_t* u, const uint8_t* v, int w, int h, int qp, int ctu_log2,
                             uint32_t opts, void* cus, int16_t* levels, uint64_t* num_levels, uint8_t* ry,
                             uint8_t* ru, uint8_t* rv) {
  return orc::mt_encode(y, u, v, w, h, qp, ctu_log2, opts, (vvcg_cu_rec*)cus, levels, num_levels, ry, ru, rv);
}
extern "C" int orc_mt_decode(const void* cus, const int16_t* levels, uint64_t num_levels, int w, int h, int qp,
                             int ctu_log2, uint32_t opts, uint8_t* ry, uint8_t* ru, uint8_t* rv) {
  return orc::mt_decode((const vvcg_cu_rec*)cus, levels, num_levels, w, h, qp, ctu_log2, opts, ry, ru, rv);
}
extern "C" int orc_inter_encode(const uint8_t* y, const uint8_t* u, const uint8_t* v, int w, int h, int qp,
                                int ctu_log2, uint32_t opts, const uint8_t* const* refs, int num_refs, void* cus,
                                int16_t* levels, uint64_t* num_levels, uint8_t* ry, uint8_t* ru, uint8_t* rv) {
  return orc::inter_encode(y, u, v, w, h, qp, ctu_log2, opts, refs, num_refs, (vvcg_inter_cu*)cus, levels, num_levels,
                           ry, ru, rv);
}
extern "C" int orc_inter_resolve_motion(void* cus, int w, int h, int ctu_log2) {
  return orc::inter_resolve_motion((vvcg_inter_cu*)cus, w, h, ctu_log2);
}
extern "C" int orc_inter_decode(const void* cus, const int16_t* levels, uint64_t num_levels, int w, int h, int qp,
                                int ctu_log2, uint32_t opts, const uint8_t* const* refs, int num_refs, uint8_t* ry,
                                uint8_t* ru, uint8_t* rv) {
  return orc::inter_decode((const vvcg_inter_cu*)cus, levels, num_levels, w, h, qp, ctu_log2, opts, refs, num_refs,
                           ry, ru, rv);
}
extern "C" void orc_derive_intra_mpms(int left, int above, uint8_t* mpm) { orc::derive_intra_mpms(left, above, mpm); }
extern "C" int orc_mt_write(const void* cus, const int16_t* levels, uint64_t num_levels, int w, int h, int qp,
                            uint32_t opts, uint8_t* out, uint64_t cap, uint64_t* size) {
  std::vector<uint8_t> b;
  const int rc = orc::mt_write((const vvcg_cu_rec*)cus, levels, num_levels, w, h, qp, opts, &b);
  if (rc) return rc;
  if (b.size() > cap) return -1000;
  memcpy(out, b.data(), b.size());
  *size = b.size();
  return 0;
}
extern "C" int orc_p_write(const void* cus, const int16_t* levels, uint64_t num_levels, int w, int h, int qp,
                           uint32_t opts, uint8_t* out, uint64_t cap, uint64_t* size) {
  std::vector<uint8_t> b;
  const int rc = orc::p_write((const vvcg_inter_cu*)cus, levels, num_levels, w, h, qp, opts, &b);
  if (rc) return rc;
  if (b.size() > cap) return -1000;
  memcpy(out, b.data(), b.size());
  *size = b.size();
  return 0;
}
