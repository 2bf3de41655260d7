// Host-side H.266 bitstream assembly around the slice data: RBSP bit
// writing, emulation prevention, Annex-B NAL framing, the parameter sets,
// picture header and slice header the reference encoder writes for its
// default (8-bit 4:2:0, 32x32 CTU) stream, and the reverse: an Annex-B
// access unit split into NAL units and the slice data found in it.
//
// Follows crates/rustmpeg-video/src/vvc: bits.rs:21-142 (BitWriter),
// :231-266 (rbsp_to_ebsp / ebsp_to_rbsp); hls.rs:182-206 (select_level_idc),
// :220-346 (profile_tier_level and general_constraints_info), :353-365
// (VPS), :373-499 (SPS), :501-522 (VUI payload), :529-564 (PPS), :571-586
// (picture header), :598-637 (slice header), :756-770 (AUD, push_nal);
// mod.rs:490-536 and :582-616 (the encoder's stream configuration and the
// order of the NAL units in an IDR access unit). The syntax order is the
// H.266 specification's, so it is the reference's.
#pragma once
#include <stdint.h>
#include <stddef.h>

#include <vector>

namespace vvcg {
namespace annexb {

// NAL unit types (H.266 Table 5)
constexpr uint8_t kNalIdrNLp = 8, kNalVps = 14, kNalSps = 15, kNalPps = 16, kNalPh = 19, kNalAud = 20;

struct StreamCfg {  // the reference's VvcStreamConfig
  uint32_t width, height, crop_right, crop_bottom;
  uint8_t qp, level_idc, ctu_log2, min_cb_log2, ts_log2;
};

class Bits {  // MSB first
 public:
  std::vector<uint8_t> out;
  void bit(bool b) {
    acc_ = (uint8_t)((acc_ << 1) | (b ? 1 : 0));
    if (++n_ == 8) {
      out.push_back(acc_);
      acc_ = 0;
      n_ = 0;
    }
  }
  void u(uint32_t v, int n) {
    for (int i = n - 1; i >= 0; i--) bit((v >> i) & 1u);
  }
  void ue(uint64_t v) {  // Exp-Golomb of v: (len - 1) zeros, then v + 1 in len bits
    const uint64_t x = v + 1;
    int len = 0;
    while ((x >> len) > 1) len++;
    for (int i = 0; i < len; i++) bit(false);
    for (int i = len; i >= 0; i--) bit((x >> i) & 1u);
  }
  void se(int32_t v) { ue(v > 0 ? 2 * (uint64_t)v - 1 : 2 * (uint64_t)(-(int64_t)v)); }
  bool aligned() const { return n_ == 0; }
  void zero_align() {
    while (n_) bit(false);
  }
  void one_then_align() {  // rbsp_trailing_bits() and byte_alignment()
    bit(true);
    zero_align();
  }
  void bytes(const uint8_t* p, size_t n) { out.insert(out.end(), p, p + n); }  // byte-aligned only

 private:
  uint8_t acc_ = 0;
  int n_ = 0;
};

inline uint8_t level_idc_for(uint32_t w, uint32_t h) {
  // (level_idc, maximum luma samples per picture), H.266 Table A.1
  static const struct { uint8_t idc; uint64_t max; } kLevels[] = {
      {16, 36864},    {32, 122880},   {35, 245760},   {48, 552960},   {51, 983040},
      {64, 2228224},  {67, 2228224},  {80, 8912896},  {83, 8912896},  {86, 8912896},
      {96, 35651584}, {99, 35651584}, {102, 35651584}};
  const uint64_t s = (uint64_t)w * h;
  for (const auto& l : kLevels)
    if (s <= l.max) return l.idc;
  return 102;
}

// profile_tier_level(1, 0) with the general constraints the intra-only
// default tool set implies (MTS, LFNST and transform skip allowed).
inline void write_ptl(Bits& b, uint8_t level_idc, uint8_t ctu_log2) {
  b.u(1, 7);  // general_profile_idc: Main 10
  b.bit(false);  // general_tier_flag
  b.u(level_idc, 8);
  b.bit(true);   // ptl_frame_only_constraint_flag
  b.bit(false);  // ptl_multilayer_enabled_flag
  // general_constraints_info(): present; the flags in syntax order
  b.bit(true);                                       // gci_present_flag
  b.bit(true); b.bit(true); b.bit(false);            // intra only, all layers independent, one AU only
  b.u(8, 4); b.u(2, 2);                              // max bit depth 8, max chroma format 4:2:0
  b.bit(true); b.bit(true); b.bit(true); b.bit(true); b.bit(true);  // mixed NALU types, TRAIL, STSA, RASL, RADL
  b.bit(false); b.bit(true); b.bit(true); b.bit(false); b.bit(true);  // IDR, CRA, GDR, APS, IDR RPL
  b.bit(true); b.bit(false); b.bit(true); b.bit(false); b.bit(false); b.bit(true);  // tiles, PH in SH, slices, subpics
  const uint8_t c = ctu_log2 < 5 ? 5 : ctu_log2 > 7 ? 7 : ctu_log2;
  b.u(8u - c, 2);                                    // three_minus_max_log2_ctu_size
  b.bit(true); b.bit(true); b.bit(true);             // partition override, MTT, dual tree
  b.bit(true); b.bit(true); b.bit(true); b.bit(true); b.bit(true); b.bit(true);  // palette IBC ISP MRL MIP CCLM
  for (int i = 0; i < 16; i++) b.bit(true);          // the 16 inter-tool constraints
  b.bit(true);   // no luma transform size 64
  b.bit(false);  // transform skip allowed
  b.bit(true);   // no BDPCM
  b.bit(false); b.bit(false);                        // MTS, LFNST allowed
  b.bit(true); b.bit(true); b.bit(true); b.bit(true);  // joint CbCr, SBT, ACT, explicit scaling lists
  b.bit(true); b.bit(true); b.bit(true); b.bit(true);  // dependent quantisation, sign hiding, CU QP delta, chroma QP offset
  for (int i = 0; i < 6; i++) b.bit(true);           // SAO ALF CCALF LMCS LADF virtual boundaries
  b.u(0, 8);     // gci_num_additional_bits
  b.zero_align();
  b.zero_align();  // ptl_reserved_zero_bit (no sub-layers)
  b.u(0, 8);       // ptl_num_sub_profiles
}

inline std::vector<uint8_t> vps_rbsp(const StreamCfg& c) {
  Bits b;
  b.u(1, 4);  // vps_video_parameter_set_id
  b.u(0, 6);  // vps_max_layers_minus1
  b.u(0, 3);  // vps_max_sublayers_minus1
  b.u(0, 6);  // vps_layer_id[0]
  b.zero_align();
  write_ptl(b, c.level_idc, c.ctu_log2);
  b.bit(false);  // vps_extension_flag
  b.one_then_align();
  return b.out;
}

inline std::vector<uint8_t> vui_payload() {
  Bits b;
  b.bit(true); b.bit(false); b.bit(true); b.bit(true);  // progressive, interlaced, non-packed, non-projected
  b.bit(false); b.bit(false);                           // aspect ratio, overscan
  b.bit(true); b.u(1, 8); b.u(1, 8); b.u(1, 8);         // colour description: BT.709 primaries, transfer, matrix
  b.bit(false);                                         // full range
  b.bit(true); b.ue(0);                                 // chroma sample location type 0
  b.one_then_align();
  return b.out;
}

// The SPS of the default tool set (8-bit 4:2:0; MTS, LFNST and transform
// skip enabled; everything else off); returns an empty vector for a CTU
// size the syntax cannot signal.
inline std::vector<uint8_t> sps_rbsp(const StreamCfg& c) {
  if (c.ctu_log2 < 5 || c.ctu_log2 > 7 || c.min_cb_log2 < 2 || c.ts_log2 < 2) return {};
  Bits b;
  b.u(0, 4);  // sps_seq_parameter_set_id
  b.u(1, 4);  // sps_video_parameter_set_id
  b.u(0, 3);  // sps_max_sub_layers_minus1
  b.u(1, 2);  // sps_chroma_format_idc: 4:2:0
  b.u(c.ctu_log2 - 5u, 2);
  b.bit(true);  // sps_ptl_dpb_hrd_params_present_flag
  write_ptl(b, c.level_idc, c.ctu_log2);
  b.bit(false); b.bit(false);  // GDR, reference picture resampling
  b.ue(c.width);
  b.ue(c.height);
  const bool crop = c.crop_right || c.crop_bottom;
  b.bit(crop);  // sps_conformance_window_flag, offsets in chroma samples
  if (crop) {
    b.ue(0); b.ue(c.crop_right / 2); b.ue(0); b.ue(c.crop_bottom / 2);
  }
  b.bit(false);  // sps_subpic_info_present_flag
  b.ue(0);       // sps_bitdepth_minus8
  b.bit(false); b.bit(false);  // entropy coding sync, entry point offsets
  b.u(4, 4);     // sps_log2_max_pic_order_cnt_lsb_minus4
  b.bit(false);  // sps_poc_msb_cycle_flag
  b.u(0, 2); b.u(0, 2);  // extra PH / SH bytes
  b.ue(0); b.ue(0); b.ue(0);  // dpb_parameters: max dec pic buffering, reorder, latency
  b.ue(c.min_cb_log2 - 2u);
  b.bit(false);  // sps_partition_constraints_override_enabled_flag
  b.ue(0); b.ue(0);  // intra slice luma: min QT diff, max MTT depth
  b.bit(false);      // sps_qtbtt_dual_tree_intra_flag
  b.ue(0); b.ue(0);  // inter slice: min QT diff, max MTT depth
  if (c.ctu_log2 > 5) b.bit(false);  // sps_max_luma_transform_size_64_flag
  b.bit(true);                // sps_transform_skip_enabled_flag
  b.ue(c.ts_log2 - 2u);       // sps_log2_transform_skip_max_size_minus2
  b.bit(false);               // sps_bdpcm_enabled_flag
  b.bit(true); b.bit(true); b.bit(false);  // MTS; explicit MTS intra, inter
  b.bit(true);                // sps_lfnst_enabled_flag
  b.bit(false);               // sps_joint_cbcr_enabled_flag
  b.bit(true);                // sps_same_qp_table_for_chroma_flag
  b.se(0); b.ue(0); b.ue(0); b.ue(0);  // the one-point chroma QP table
  b.bit(false); b.bit(false);  // SAO, ALF
  b.bit(false); b.bit(false); b.bit(false);  // LMCS, weighted pred, weighted bipred
  b.bit(false); b.bit(false);  // long-term refs, inter-layer prediction
  b.bit(false); b.bit(true);   // IDR RPL present, RPL1 same as RPL0
  b.ue(0);                     // sps_num_ref_pic_lists[0]
  for (int i = 0; i < 7; i++) b.bit(false);  // wraparound TMVP AMVR BDOF SMVD DMVR MMVD
  b.ue(5);                     // sps_six_minus_max_num_merge_cand
  for (int i = 0; i < 4; i++) b.bit(false);  // SBT affine BCW CIIP
  b.ue(0);                     // sps_log2_parallel_merge_level_minus2
  for (int i = 0; i < 7; i++) b.bit(false);  // ISP MRL MIP CCLM, chroma collocation h / v, palette
  b.ue(0);                     // sps_internal_bit_depth_minus_input_bit_depth
  for (int i = 0; i < 8; i++) b.bit(false);  // IBC LADF scaling lists DQ SDH virtual boundaries HRD field seq
  b.bit(true);                 // sps_vui_parameters_present_flag
  const std::vector<uint8_t> vui = vui_payload();
  b.ue(vui.size() - 1);
  b.zero_align();
  b.bytes(vui.data(), vui.size());
  b.bit(false);  // sps_extension_present_flag
  b.one_then_align();
  return b.out;
}

inline std::vector<uint8_t> pps_rbsp(const StreamCfg& c) {
  Bits b;
  b.u(0, 6); b.u(0, 4);  // PPS id, SPS id
  b.bit(false);          // pps_mixed_nalu_types_in_pic_flag
  b.ue(c.width);
  b.ue(c.height);
  b.bit(false); b.bit(false); b.bit(false);  // conformance window, scaling window, output flag
  b.bit(true);                 // pps_no_pic_partition_flag
  b.bit(false); b.bit(false);  // subpic id mapping, CABAC init present
  b.ue(0); b.ue(0);            // default active ref idx L0 / L1
  for (int i = 0; i < 4; i++) b.bit(false);  // RPL1 idx, weighted pred / bipred, wraparound
  b.se((int32_t)c.qp - 26);    // pps_init_qp_minus26
  b.bit(false); b.bit(false);  // CU QP delta, chroma tool offsets
  b.bit(true);                 // pps_deblocking_filter_control_present_flag
  b.bit(false);                // pps_deblocking_filter_override_enabled_flag
  b.bit(true);                 // pps_deblocking_filter_disabled_flag
  b.bit(false); b.bit(false); b.bit(false);  // PH / SH extensions, pps_extension_flag
  b.one_then_align();
  return b.out;
}

inline std::vector<uint8_t> ph_rbsp(uint32_t poc_lsb) {
  Bits b;
  b.bit(true); b.bit(false); b.bit(false); b.bit(false);  // IRAP, non-ref, GDR, inter slices allowed
  b.ue(0);                // ph_pic_parameter_set_id
  b.u(poc_lsb & 0xFF, 8); // ph_pic_order_cnt_lsb
  b.one_then_align();
  return b.out;
}

// The IDR slice header of the default tool set, byte-aligned (the slice
// data follows it in the same NAL unit).
inline std::vector<uint8_t> slice_header(int32_t qp_delta) {
  Bits b;
  b.bit(false); b.bit(false);  // PH in SH, no output of prior pictures
  b.se(qp_delta);              // sh_qp_delta
  b.bit(false);                // sh_ts_residual_coding_disabled_flag
  b.one_then_align();          // byte_alignment()
  return b.out;
}

inline std::vector<uint8_t> aud_rbsp(uint8_t pic_type) {
  Bits b;
  b.bit(true);  // aud_irap_or_gdr_au_flag
  b.u(pic_type & 7u, 3);
  b.one_then_align();
  return b.out;
}

// A 0x03 before every byte <= 3 that follows two zero bytes.
inline void append_escaped(std::vector<uint8_t>& out, const uint8_t* rbsp, size_t n) {
  int zeros = 0;
  for (size_t i = 0; i < n; i++) {
    if (zeros >= 2 && rbsp[i] <= 3) {
      out.push_back(3);
      zeros = 0;
    }
    out.push_back(rbsp[i]);
    zeros = rbsp[i] == 0 ? zeros + 1 : 0;
  }
}

inline std::vector<uint8_t> unescape(const uint8_t* p, size_t n) {
  std::vector<uint8_t> r;
  r.reserve(n);
  for (size_t i = 0; i < n;) {
    if (i + 2 < n && p[i] == 0 && p[i + 1] == 0 && p[i + 2] == 3) {
      r.push_back(0);
      r.push_back(0);
      i += 3;
    } else {
      r.push_back(p[i++]);
    }
  }
  return r;
}

// Start code, the two-byte NAL unit header (layer 0, TemporalId 0), escaped RBSP.
inline void push_nal(std::vector<uint8_t>& out, uint8_t type, const std::vector<uint8_t>& rbsp) {
  const uint8_t hdr[6] = {0, 0, 0, 1, 0, (uint8_t)(((type & 0x1F) << 3) | 1)};
  out.insert(out.end(), hdr, hdr + 6);
  append_escaped(out, rbsp.data(), rbsp.size());
}

// The encoder's stream configuration for a visible picture: coded size
// padded to whole 32x32 CTUs, the rest as conformance-window crop.
inline StreamCfg encoder_cfg(uint32_t width, uint32_t height, uint8_t qp) {
  StreamCfg c{};
  c.width = (width + 31) & ~31u;
  c.height = (height + 31) & ~31u;
  c.crop_right = c.width - width;
  c.crop_bottom = c.height - height;
  c.qp = qp;
  c.level_idc = level_idc_for(c.width, c.height);
  c.ctu_log2 = 5;
  c.min_cb_log2 = 5;
  c.ts_log2 = 5;
  return c;
}

// One IDR access unit: AUD, VPS, SPS, PPS, PH (POC 0), then the IDR_N_LP
// slice (header at slice QP delta 0, then the slice data).
inline std::vector<uint8_t> idr_access_unit(const StreamCfg& c, const uint8_t* slice_data, size_t n) {
  std::vector<uint8_t> au;
  au.reserve(n + n / 64 + 256);
  push_nal(au, kNalAud, aud_rbsp(0));
  push_nal(au, kNalVps, vps_rbsp(c));
  push_nal(au, kNalSps, sps_rbsp(c));
  push_nal(au, kNalPps, pps_rbsp(c));
  push_nal(au, kNalPh, ph_rbsp(0));
  std::vector<uint8_t> slice = slice_header(0);
  slice.insert(slice.end(), slice_data, slice_data + n);
  push_nal(au, kNalIdrNLp, slice);
  return au;
}

struct Nal {
  uint8_t type, layer, tid_plus1;
  size_t begin, end;  // the escaped payload after the two-byte header, in the access unit
};

// The NAL units of an Annex-B byte stream (3- or 4-byte start codes;
// trailing zero bytes before a start code belong to no NAL unit).
inline std::vector<Nal> split(const uint8_t* p, size_t n) {
  std::vector<size_t> starts;  // first byte after each start code
  for (size_t i = 0; i + 2 < n; i++)
    if (p[i] == 0 && p[i + 1] == 0 && p[i + 2] == 1) {
      starts.push_back(i + 3);
      i += 2;
    }
  std::vector<Nal> nals;
  for (size_t k = 0; k < starts.size(); k++) {
    size_t end = k + 1 < starts.size() ? starts[k + 1] - 3 : n;
    while (end > starts[k] && p[end - 1] == 0) end--;
    if (end < starts[k] + 2) continue;
    const uint8_t* h = p + starts[k];
    nals.push_back(Nal{(uint8_t)(h[1] >> 3), (uint8_t)(h[0] & 0x3F), (uint8_t)(h[1] & 7), starts[k] + 2, end});
  }
  return nals;
}

class Reader {  // MSB first over an unescaped RBSP
 public:
  Reader(const uint8_t* p, size_t n) : p_(p), n_(n) {}
  bool ok() const { return ok_; }
  size_t pos() const { return pos_; }
  uint32_t u(int n) {
    uint32_t v = 0;
    for (int i = 0; i < n; i++) {
      if (pos_ >= n_ * 8) {
        ok_ = false;
        return 0;
      }
      v = (v << 1) | ((p_[pos_ >> 3] >> (7 - (pos_ & 7))) & 1u);
      pos_++;
    }
    return v;
  }
  uint32_t ue() {
    int z = 0;
    while (ok_ && u(1) == 0)
      if (++z > 31) ok_ = false;
    return ok_ ? (uint32_t)(((1ull << z) - 1) + u(z)) : 0;
  }
  int32_t se() {
    const uint32_t k = ue();
    return (k & 1) ? (int32_t)((k + 1) / 2) : -(int32_t)(k / 2);
  }

 private:
  const uint8_t* p_;
  size_t n_, pos_ = 0;
  bool ok_ = true;
};

}  // namespace annexb
}  // namespace vvcg
