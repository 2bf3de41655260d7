// The general decoder's picture pass over a batch of intra pictures
// (vvcg_gen_prepare / vvcg_gen_run / vvcg_gen_download): host side. Included
// at the end of vvcg.cu (it uses the context and the transform-unit tables
// defined there).
//
// Per run: the residual slots are cleared and every coded block's residual
// is computed by the size-binned TU kernels; the intra reconstruction runs
// level by level (k_gen_recon_level), each level a launch over the groups of
// every picture that have no dependency left; then per picture the general
// deblocking (two launches), SAO (one per component) and ALF (two launches).
//
// Dependency levels (host, at prepare): the groups of a picture are visited
// in decode order over a 4x4 luma cell grid holding, per cell, the highest
// level of a group whose blocks cover it (area) and of a group that may read
// it (read). A group may read samples up to 4 to the left of and above its
// bounding box and up to twice its width to the right and its height below
// (above-right / below-left references, MRL lines, ISP and CCLM templates).
// Its level is one above the highest area level over its read and own boxes
// (the samples it reads, and the luma a chroma-only group's CCLM reads) and
// the highest read level over its own box (earlier groups that read where
// it writes must have read first).

namespace {

struct GenPicLayout {
  uint64_t plane_off[2][3];  // samples, in GenPass::planes: set 0 (reconstruction), set 1
  uint32_t stride[3];
  uint64_t dy_off, dc_off;   // bytes, in GenPass::maps
  int final_set;             // the set holding the output
  uint32_t ctu_cols, ctu_rows;
};

}  // namespace

struct GenPass {
  bool prepared = false;
  std::vector<vvcg_gen_pic> pics;
  std::vector<GenPicLayout> lay;
  std::vector<uint32_t> level_start;  // levels + 1 offsets into the level-ordered groups
  uint32_t tu_count[kTuBins] = {0, 0, 0};
  uint64_t slot_count = 0, maps_bytes = 0;
  DevBuf planes, maps, states, reqs, tus, tu_idx, group_first, group_pic, level_groups, levels, res, pred, cells,
      ccells, sao, alf_ctus, alf_params;
  std::vector<DbkGenArgs> dbk;          // per picture (pictures without deblocking: unused)
  std::vector<SaoBoundedPass> sao_pass;  // 3 per picture with SAO
  std::vector<AlfGenPass> alf_pass;      // per picture with ALF
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  uint32_t graph_launches = 0;
  void drop_graph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
  }
  void release() {
    drop_graph();
    for (DevBuf* b : {&planes, &maps, &states, &reqs, &tus, &tu_idx, &group_first, &group_pic, &level_groups, &levels,
                      &res, &pred, &cells, &ccells, &sao, &alf_ctus, &alf_params})
      b->release();
  }
};

void gen_pass_free(GenPass* g) {
  if (!g) return;
  g->release();
  delete g;
}

namespace {

template <class T>
vvcg_status gen_upload(vvcg_ctx* ctx, DevBuf& b, const T* src, size_t n) {
  CK(b.reserve(std::max<size_t>(1, n) * sizeof(T)), "cudaMalloc");
  if (n) CK(cudaMemcpyAsync(b.p, src, n * sizeof(T), cudaMemcpyHostToDevice, ctx->stream), "upload");
  return VVCG_OK;
}

// mark_tu (decode_general.rs:4837-4907) of one block into the picture's
// deblocking maps: the transform block's id and size over the luma 4x4 cells
// or chroma 2x2 cells its samples touch, the luma cbf, and the coded / intra
// flags of the intra coding unit.
void gen_mark(const vvcg_gen_tb& t, uint32_t id, uint32_t cols, uint32_t rows, vvcg_dbk_cell* cells,
              uint32_t ccols, uint32_t crows, vvcg_dbk_ccell* cc) {
  const vvcg_gen_intra_req& r = t.pred;
  if (r.comp == 0) {
    const uint32_t x1 = std::min<uint32_t>(r.x + r.w, cols * 4), y1 = std::min<uint32_t>(r.y + r.h, rows * 4);
    for (uint32_t cy = r.y / 4; cy < (y1 + 3) / 4; cy++)
      for (uint32_t cx = r.x / 4; cx < (x1 + 3) / 4; cx++) {
        vvcg_dbk_cell& c = cells[(size_t)cy * cols + cx];
        c.tu_id = id;
        c.tu_w = r.w;
        c.tu_h = r.h;
        c.flags = (uint8_t)((c.flags & ~VVCG_DBK_CBF) | (t.coded ? VVCG_DBK_CBF : 0));
      }
    // the coding unit's LumaCell fields: intra, valid
    const uint32_t cx1 = std::min<uint32_t>(r.cu_x + r.cu_w, cols * 4), cy1 = std::min<uint32_t>(r.cu_y + r.cu_h, rows * 4);
    for (uint32_t cy = r.cu_y / 4; cy < (cy1 + 3) / 4; cy++)
      for (uint32_t cx = r.cu_x / 4; cx < (cx1 + 3) / 4; cx++)
        cells[(size_t)cy * cols + cx].flags |= VVCG_DBK_CODED | VVCG_DBK_INTRA;
  } else {
    const uint32_t x1 = std::min<uint32_t>(r.x + r.w, ccols * 2), y1 = std::min<uint32_t>(r.y + r.h, crows * 2);
    for (uint32_t cy = r.y / 2; cy < (y1 + 1) / 2; cy++)
      for (uint32_t cx = r.x / 2; cx < (x1 + 1) / 2; cx++) {
        vvcg_dbk_ccell& c = cc[(size_t)cy * ccols + cx];
        (r.comp == 1 ? c.tu_cb : c.tu_cr) = id;
        c.tu_w = r.w;
        c.tu_h = r.h;
      }
  }
}

const char* gen_pic_error(const vvcg_gen_pic& p, const vvcg_gen_batch* b) {
  const uint32_t ctu = 1u << p.ctu_log2;
  if (p.ctu_log2 < 4 || p.ctu_log2 > 7) return "CTU size outside 16..128";
  if (!p.width || !p.height || p.width % ctu || p.height % ctu || (p.width & 7) || (p.height & 7))
    return "coded size not whole CTUs";
  if (p.width > 16384 || p.height > 16384) return "coded size above 16384";
  if (!p.vis_width || !p.vis_height || p.vis_width > p.width || p.vis_height > p.height) return "visible size";
  if (p.bit_depth < 8 || p.bit_depth > 12) return "bit depth";
  if (p.tools & ~(uint32_t)(VVCG_TOOL_DEBLOCK | VVCG_TOOL_SAO | VVCG_TOOL_ALF)) return "tools";
  if ((uint64_t)p.group_offset + p.num_groups > b->num_groups) return "groups out of range";
  const uint64_t nctu = (uint64_t)((p.vis_width + ctu - 1) / ctu) * ((p.vis_height + ctu - 1) / ctu);
  if ((p.tools & VVCG_TOOL_SAO) && (!b->sao || (uint64_t)p.sao_offset + 3 * nctu > b->num_sao))
    return "SAO parameters out of range";
  if (p.tools & VVCG_TOOL_ALF) {
    if (!b->alf_ctus || (uint64_t)p.alf_offset + nctu > b->num_alf_ctus) return "ALF CTU switches out of range";
    if (p.alf_params < 0 || (uint32_t)p.alf_params >= b->num_alf_params || !b->alf_params) return "ALF parameters";
    const vvcg_alf_params& a = b->alf_params[p.alf_params];
    if (a.num_luma_filters > 25 || a.num_chroma_filters > 8 || a.num_cc_cb > 4 || a.num_cc_cr > 4)
      return "ALF filter counts";
    for (uint64_t k = 0; k < nctu; k++) {
      const vvcg_alf_ctu& m = b->alf_ctus[p.alf_offset + k];
      if (m.luma_mode > VVCG_ALF_APS || (m.luma_mode == VVCG_ALF_APS && a.num_luma_filters == 0))
        return "ALF CTU luma mode";
    }
  }
  if ((p.tools & VVCG_TOOL_DEBLOCK) &&
      (p.dbk.num_ref[0] < 0 || p.dbk.num_ref[0] > 16 || p.dbk.num_ref[1] < 0 || p.dbk.num_ref[1] > 16))
    return "deblocking reference list lengths";
  return nullptr;
}

}  // namespace

extern "C" {

uint32_t vvcg_gen_levels(const vvcg_ctx* ctx) {
  return ctx && ctx->gen && ctx->gen->prepared ? (uint32_t)ctx->gen->level_start.size() - 1 : 0;
}

vvcg_status vvcg_gen_prepare(vvcg_ctx* ctx, const vvcg_gen_batch* b) {
  if (!ctx) return VVCG_INVALID_INPUT;
  if (!ctx->gen) ctx->gen = new GenPass();
  GenPass& G = *ctx->gen;
  G.prepared = false;
  G.drop_graph();
  if (!b || !b->pics || !b->num_pics) return fail(ctx, VVCG_INVALID_INPUT, "empty batch");
  if (!b->group_first || (b->num_tbs && !b->tbs)) return fail(ctx, VVCG_INVALID_INPUT, "missing blocks or groups");
  if (b->num_tbs > (1u << 30) || b->num_groups > (1u << 30)) return fail(ctx, VVCG_LIMIT_EXCEEDED, "too many blocks");
  for (uint32_t g = 0; g < b->num_groups; g++)
    if (b->group_first[g] > b->group_first[g + 1]) return fail(ctx, VVCG_INVALID_INPUT, "group %u: decreasing", g);
  if (b->group_first[b->num_groups] > b->num_tbs) return fail(ctx, VVCG_INVALID_INPUT, "groups past the blocks");
  if (b->num_levels && !b->levels) return fail(ctx, VVCG_INVALID_INPUT, "missing levels");
  CK(cudaSetDevice(ctx->device), "cudaSetDevice");
  CK(cudaStreamSynchronize(ctx->stream), "prepare");
  const uint32_t np = b->num_pics;
  G.pics.assign(b->pics, b->pics + np);
  G.lay.assign(np, GenPicLayout{});
  G.slot_count = b->slot_count;

  // -- pictures: layout, states, validation of their blocks ------------------
  std::vector<uint32_t> group_pic(b->num_groups, UINT32_MAX);
  uint64_t samples = 0, maps = 0, cells_n = 0, ccells_n = 0;
  for (uint32_t i = 0; i < np; i++) {
    const vvcg_gen_pic& p = G.pics[i];
    if (const char* e = gen_pic_error(p, b)) return fail(ctx, VVCG_INVALID_INPUT, "picture %u: %s", i, e);
    GenPicLayout& L = G.lay[i];
    const uint32_t ctu = 1u << p.ctu_log2;
    L.ctu_cols = (p.vis_width + ctu - 1) / ctu;
    L.ctu_rows = (p.vis_height + ctu - 1) / ctu;
    for (int c = 0; c < 3; c++) {
      const uint32_t w = c ? p.width / 2 : p.width, h = c ? p.height / 2 : p.height;
      L.stride[c] = (w + 63) & ~63u;
      for (int s = 0; s < 2; s++) {
        L.plane_off[s][c] = samples;
        samples += (uint64_t)L.stride[c] * h;
      }
    }
    L.dy_off = maps;
    maps += (uint64_t)(p.width / 4) * (p.height / 4);
    L.dc_off = maps;
    maps += (uint64_t)(p.width / 2) * (p.height / 2);
    maps = (maps + 255) & ~255ull;
    cells_n += (uint64_t)(p.width / 4) * (p.height / 4);
    ccells_n += (uint64_t)(p.width / 4) * (p.height / 4);
    for (uint32_t g = p.group_offset; g < p.group_offset + p.num_groups; g++) {
      if (group_pic[g] != UINT32_MAX) return fail(ctx, VVCG_INVALID_INPUT, "group %u in two pictures", g);
      group_pic[g] = i;
    }
  }
  for (uint32_t g = 0; g < b->num_groups; g++)
    if (group_pic[g] == UINT32_MAX && b->group_first[g] != b->group_first[g + 1])
      return fail(ctx, VVCG_INVALID_INPUT, "group %u belongs to no picture", g);
  CK(G.planes.reserve(std::max<uint64_t>(1, samples) * sizeof(uint16_t)), "cudaMalloc");
  CK(G.maps.reserve(std::max<uint64_t>(1, maps)), "cudaMalloc");
  G.maps_bytes = maps;
  uint16_t* base = (uint16_t*)G.planes.p;
  uint8_t* mbase = (uint8_t*)G.maps.p;
  std::vector<vvcg_gen_intra_state> states(np);
  for (uint32_t i = 0; i < np; i++) {
    const vvcg_gen_pic& p = G.pics[i];
    const GenPicLayout& L = G.lay[i];
    vvcg_gen_intra_state& S = states[i];
    memset(&S, 0, sizeof(S));
    for (int c = 0; c < 3; c++) {
      S.plane[c] = base + L.plane_off[0][c];
      S.stride[c] = L.stride[c];
    }
    S.width = p.width;
    S.height = p.height;
    S.dec_y = mbase + L.dy_off;
    S.dec_c = mbase + L.dc_off;
    S.bit_depth = p.bit_depth;
    S.vert_collocated = p.vert_collocated;
    S.ctu_size = 1u << p.ctu_log2;
  }

  // -- blocks: validation, coded blocks by size bin, slot overlap ------------
  const uint64_t ntb = b->group_first[b->num_groups];
  std::vector<vvcg_gen_intra_req> reqs(ntb);
  std::vector<vvcg_tu_rec> tus;
  std::vector<std::pair<uint32_t, uint32_t>> slots;  // (out_off, end) per block
  slots.reserve(ntb);
  for (uint32_t g = 0; g < b->num_groups; g++) {
    if (b->group_first[g] == b->group_first[g + 1]) continue;
    const vvcg_gen_pic& p = G.pics[group_pic[g]];
    for (uint32_t q = b->group_first[g]; q < b->group_first[g + 1]; q++) {
      const vvcg_gen_tb& t = b->tbs[q];
      if (const char* e = gen_intra_req_error(&states[group_pic[g]], t.pred, b->slot_count))
        return fail(ctx, VVCG_INVALID_INPUT, "block %u: %s", q, e);
      if (t.pred.comp && (t.pred.w < 2 || t.pred.h < 2)) return fail(ctx, VVCG_INVALID_INPUT, "block %u: chroma", q);
      reqs[q] = t.pred;
      slots.emplace_back(t.pred.out_off, t.pred.out_off + (uint32_t)t.pred.w * t.pred.h);
      if (!t.coded) continue;
      const vvcg_tu_rec& r = t.tu;
      if ((1u << r.log2_w) != t.pred.w || (1u << r.log2_h) != t.pred.h || r.out_off != t.pred.out_off ||
          r.bit_depth != p.bit_depth)
        return fail(ctx, VVCG_INVALID_INPUT, "block %u: residual record does not match the block", q);
      if (const char* why = tu_reject(r, false, b->num_levels, b->slot_count))
        return fail(ctx, VVCG_INVALID_INPUT, "block %u: %s", q, why);
      tus.push_back(r);
    }
  }
  std::sort(slots.begin(), slots.end());
  for (size_t k = 1; k < slots.size(); k++)
    if (slots[k].first < slots[k - 1].second) return fail(ctx, VVCG_INVALID_INPUT, "blocks share residual slots");
  for (int k = 0; k < kTuBins; k++) G.tu_count[k] = 0;
  for (const vvcg_tu_rec& r : tus) G.tu_count[tu_bin(r)]++;
  std::vector<uint32_t> tu_idx(tus.size());
  {
    uint32_t at[kTuBins] = {0, G.tu_count[0], G.tu_count[0] + G.tu_count[1]};
    for (uint32_t k = 0; k < (uint32_t)tus.size(); k++) tu_idx[at[tu_bin(tus[k])]++] = k;
  }

  // -- dependency levels ------------------------------------------------------
  std::vector<uint32_t> group_level(b->num_groups, 0);
  uint32_t max_level = 0;
  for (uint32_t i = 0; i < np; i++) {
    const vvcg_gen_pic& p = G.pics[i];
    const int cw = (int)p.width / 4, chh = (int)p.height / 4;
    std::vector<uint32_t> area((size_t)cw * chh, 0), read((size_t)cw * chh, 0);
    for (uint32_t g = p.group_offset; g < p.group_offset + p.num_groups; g++) {
      if (b->group_first[g] == b->group_first[g + 1]) continue;
      int x0 = INT32_MAX, y0 = INT32_MAX, x1 = 0, y1 = 0;  // luma box of the group's blocks
      for (uint32_t q = b->group_first[g]; q < b->group_first[g + 1]; q++) {
        const vvcg_gen_intra_req& r = reqs[q];
        const int s = r.comp ? 2 : 1;
        x0 = std::min(x0, r.x * s);
        y0 = std::min(y0, r.y * s);
        x1 = std::max(x1, (r.x + r.w) * s);
        y1 = std::max(y1, (r.y + r.h) * s);
      }
      auto cells_of = [&](int ax0, int ay0, int ax1, int ay1, int* c) {
        c[0] = std::max(0, ax0) / 4;
        c[1] = std::max(0, ay0) / 4;
        c[2] = std::min(cw, (std::min((int)p.width, ax1) + 3) / 4);
        c[3] = std::min(chh, (std::min((int)p.height, ay1) + 3) / 4);
      };
      int own[4], rd[4];
      cells_of(x0, y0, x1, y1, own);
      cells_of(x0 - 4, y0 - 4, x0 + 2 * (x1 - x0) + 4, y0 + 2 * (y1 - y0) + 4, rd);
      uint32_t lv = 0;
      for (int cy = rd[1]; cy < rd[3]; cy++)
        for (int cx = rd[0]; cx < rd[2]; cx++) lv = std::max(lv, area[(size_t)cy * cw + cx]);
      for (int cy = own[1]; cy < own[3]; cy++)
        for (int cx = own[0]; cx < own[2]; cx++) lv = std::max(lv, read[(size_t)cy * cw + cx]);
      lv += 1;
      group_level[g] = lv;
      max_level = std::max(max_level, lv);
      for (int cy = own[1]; cy < own[3]; cy++)
        for (int cx = own[0]; cx < own[2]; cx++) area[(size_t)cy * cw + cx] = std::max(area[(size_t)cy * cw + cx], lv);
      for (int cy = rd[1]; cy < rd[3]; cy++)
        for (int cx = rd[0]; cx < rd[2]; cx++) read[(size_t)cy * cw + cx] = std::max(read[(size_t)cy * cw + cx], lv);
    }
  }
  G.level_start.assign(max_level + 1, 0);
  for (uint32_t g = 0; g < b->num_groups; g++)
    if (group_level[g]) G.level_start[group_level[g]]++;  // counts at [level]
  for (uint32_t l = 1; l <= max_level; l++) G.level_start[l] += G.level_start[l - 1];
  std::vector<uint32_t> level_groups(G.level_start[max_level]);
  {
    std::vector<uint32_t> at(G.level_start.begin(), G.level_start.end() - 1);  // level L starts at [L - 1]
    for (uint32_t g = 0; g < b->num_groups; g++)
      if (group_level[g]) level_groups[at[group_level[g] - 1]++] = g;
  }

  // -- deblocking maps (mark_tu over each picture's blocks in decode order) --
  std::vector<vvcg_dbk_cell> cells(cells_n);
  std::vector<vvcg_dbk_ccell> ccells(ccells_n);
  for (auto& c : cells) {
    memset(&c, 0, sizeof(c));
    c.tu_id = VVCG_DBK_NO_TU;
    c.ref_idx[0] = c.ref_idx[1] = -1;
  }
  for (auto& c : ccells) {
    c.tu_cb = c.tu_cr = VVCG_DBK_NO_TU;
    c.tu_w = c.tu_h = 0;
  }
  std::vector<uint64_t> cell_off(np), ccell_off(np);
  {
    uint64_t at = 0;
    for (uint32_t i = 0; i < np; i++) {
      cell_off[i] = ccell_off[i] = at;
      at += (uint64_t)(G.pics[i].width / 4) * (G.pics[i].height / 4);
    }
  }
  for (uint32_t i = 0; i < np; i++) {
    const vvcg_gen_pic& p = G.pics[i];
    const uint32_t cols = p.width / 4, rows = p.height / 4;
    uint32_t id = 0;
    if (p.num_groups)
      for (uint32_t q = b->group_first[p.group_offset]; q < b->group_first[p.group_offset + p.num_groups]; q++)
        gen_mark(b->tbs[q], id++, cols, rows, cells.data() + cell_off[i], cols, rows, ccells.data() + ccell_off[i]);
  }

  // -- uploads ------------------------------------------------------------------
  vvcg_status st;
  if ((st = gen_upload(ctx, G.states, states.data(), np)) != VVCG_OK) return st;
  if ((st = gen_upload(ctx, G.reqs, reqs.data(), reqs.size())) != VVCG_OK) return st;
  if ((st = gen_upload(ctx, G.tus, tus.data(), tus.size())) != VVCG_OK) return st;
  if ((st = gen_upload(ctx, G.tu_idx, tu_idx.data(), tu_idx.size())) != VVCG_OK) return st;
  if ((st = gen_upload(ctx, G.group_first, b->group_first, (size_t)b->num_groups + 1)) != VVCG_OK) return st;
  if ((st = gen_upload(ctx, G.group_pic, group_pic.data(), group_pic.size())) != VVCG_OK) return st;
  if ((st = gen_upload(ctx, G.level_groups, level_groups.data(), level_groups.size())) != VVCG_OK) return st;
  if ((st = gen_upload(ctx, G.levels, b->levels, b->num_levels)) != VVCG_OK) return st;
  if ((st = gen_upload(ctx, G.cells, cells.data(), cells.size())) != VVCG_OK) return st;
  if ((st = gen_upload(ctx, G.ccells, ccells.data(), ccells.size())) != VVCG_OK) return st;
  if ((st = gen_upload(ctx, G.sao, b->sao, b->sao ? b->num_sao : 0)) != VVCG_OK) return st;
  if ((st = gen_upload(ctx, G.alf_ctus, b->alf_ctus, b->alf_ctus ? b->num_alf_ctus : 0)) != VVCG_OK) return st;
  if ((st = gen_upload(ctx, G.alf_params, b->alf_params, b->alf_params ? b->num_alf_params : 0)) != VVCG_OK) return st;
  CK(G.res.reserve(std::max<uint64_t>(1, b->slot_count) * sizeof(int16_t)), "cudaMalloc");
  CK(G.pred.reserve(std::max<uint64_t>(1, b->slot_count) * sizeof(int16_t)), "cudaMalloc");

  // -- filter passes with device pointers ------------------------------------
  G.dbk.assign(np, DbkGenArgs{});
  G.sao_pass.clear();
  G.alf_pass.clear();
  for (uint32_t i = 0; i < np; i++) {
    const vvcg_gen_pic& p = G.pics[i];
    GenPicLayout& L = G.lay[i];
    const uint32_t ctu = 1u << p.ctu_log2;
    uint16_t* set[2][3];
    for (int s = 0; s < 2; s++)
      for (int c = 0; c < 3; c++) set[s][c] = base + L.plane_off[s][c];
    const int cvw = (int)(p.vis_width + 1) / 2, cvh = (int)(p.vis_height + 1) / 2;
    DbkGenArgs& A = G.dbk[i];
    for (int c = 0; c < 3; c++) {
      A.plane[c] = set[0][c];
      A.stride[c] = (int32_t)L.stride[c];
    }
    A.vis_w = (int32_t)p.vis_width;
    A.vis_h = (int32_t)p.vis_height;
    A.cw = cvw;
    A.ch = cvh;
    A.bd = p.bit_depth;
    A.ctu = (int32_t)ctu;
    A.cells = (const vvcg_dbk_cell*)G.cells.p + cell_off[i];
    A.cols = (int32_t)(p.width / 4);
    A.rows = (int32_t)(p.height / 4);
    A.cc = (const vvcg_dbk_ccell*)G.ccells.p + ccell_off[i];
    A.ccols = (int32_t)(p.width / 4);
    A.crows = (int32_t)(p.height / 4);
    A.prm = p.dbk;
    int cur = 0;
    if (p.tools & VVCG_TOOL_SAO) {
      for (int c = 0; c < 3; c++) {
        const uint32_t w = c ? p.width / 2 : p.width, h = c ? p.height / 2 : p.height;
        SaoBoundedPass S{set[0][c], set[1][c], (const vvcg_sao*)G.sao.p + p.sao_offset + (uint64_t)c * L.ctu_cols * L.ctu_rows,
                         (int32_t)L.stride[c], (int32_t)w, (int32_t)h, c ? cvw : (int32_t)p.vis_width,
                         c ? cvh : (int32_t)p.vis_height, p.bit_depth, (int32_t)(c ? ctu / 2 : ctu),
                         (int32_t)L.ctu_cols};
        G.sao_pass.push_back(S);
      }
      cur = 1;
    }
    if (p.tools & VVCG_TOOL_ALF) {
      AlfGenPass P;
      const int pw = (int)p.width, ph = (int)p.height, cw = pw / 2, ch = ph / 2;
      P.y = AlfGenView{set[cur][0], (int32_t)L.stride[0], std::min((int)p.vis_width, pw), std::min((int)p.vis_height, ph)};
      P.u = AlfGenView{set[cur][1], (int32_t)L.stride[1], std::min(cvw, cw), std::min(cvh, ch)};
      P.v = AlfGenView{set[cur][2], (int32_t)L.stride[2], std::min(cvw, cw), std::min(cvh, ch)};
      for (int c = 0; c < 3; c++) {
        P.dst[c] = set[1 - cur][c];
        P.dstride[c] = (int32_t)L.stride[c];
      }
      P.pw = pw;
      P.ph = ph;
      P.cw = cw;
      P.ch = ch;
      P.vis_w = (int)p.vis_width;
      P.vis_h = (int)p.vis_height;
      P.cvis_w = cvw;
      P.cvis_h = cvh;
      P.bd = p.bit_depth;
      P.ctu = (int)ctu;
      P.ctu_cols = (int)L.ctu_cols;
      P.ctus = (const vvcg_alf_ctu*)G.alf_ctus.p + p.alf_offset;
      P.a = (const vvcg_alf_params*)G.alf_params.p + p.alf_params;
      G.alf_pass.push_back(P);
      cur = 1 - cur;
    }
    L.final_set = cur;
  }
  G.prepared = true;
  return VVCG_OK;
}

}  // extern "C"

namespace {

// The pass of the prepared batch on the context's stream; *n counts launches.
vvcg_status gen_enqueue(vvcg_ctx* ctx, uint32_t* n) {
  GenPass& G = *ctx->gen;
  CK(cudaMemsetAsync(G.maps.p, 0, std::max<uint64_t>(1, G.maps_bytes), ctx->stream), "clear maps");
  CK(cudaMemsetAsync(G.res.p, 0, std::max<uint64_t>(1, G.slot_count) * sizeof(int16_t), ctx->stream), "clear residuals");
  uint32_t first = 0;
  for (int bin = 0; bin < kTuBins; bin++) {
    const uint32_t cnt = G.tu_count[bin];
    if (cnt) {
      const TuVariant& V = kTuTable[bin][ctx->tu_pick[0][bin]];
      V.inv<<<(cnt + V.warps - 1) / V.warps, V.warps * 32, V.smem, ctx->stream>>>(
          (const vvcg_tu_rec*)G.tus.p, (const uint32_t*)G.tu_idx.p + first, cnt, (const int16_t*)G.levels.p,
          (int16_t*)G.res.p);
      CK(cudaGetLastError(), "residual launch");
      (*n)++;
    }
    first += cnt;
  }
  const uint32_t levels = (uint32_t)G.level_start.size() - 1;
  for (uint32_t l = 0; l < levels; l++) {
    const uint32_t cnt = G.level_start[l + 1] - G.level_start[l];
    if (!cnt) continue;
    GenLevelArgs A{(const vvcg_gen_intra_state*)G.states.p, (const vvcg_gen_intra_req*)G.reqs.p,
                   (const uint32_t*)G.group_first.p, (const uint32_t*)G.group_pic.p,
                   (const uint32_t*)G.level_groups.p + G.level_start[l], cnt, (const int16_t*)G.res.p,
                   (int16_t*)G.pred.p};
    const uint32_t grid = std::min<uint32_t>((cnt + kGiWarps - 1) / kGiWarps, (uint32_t)ctx->num_sms * 8);
    k_gen_recon_level<<<grid, kGiWarps * 32, 0, ctx->stream>>>(A);
    CK(cudaGetLastError(), "intra level launch");
    (*n)++;
  }
  size_t si = 0, ai = 0;
  for (size_t i = 0; i < G.pics.size(); i++) {
    const vvcg_gen_pic& p = G.pics[i];
    if (p.tools & VVCG_TOOL_DEBLOCK) {
      const DbkGenArgs& A = G.dbk[i];
      const uint64_t cells = (uint64_t)((p.vis_width + 3) / 4) * ((p.vis_height + 3) / 4);
      const dim3 grid((uint32_t)std::min<uint64_t>((cells + 127) / 128, (uint64_t)ctx->num_sms * 16), 3);
      k_dbk_general<true><<<grid, 128, 0, ctx->stream>>>(A);
      k_dbk_general<false><<<grid, 128, 0, ctx->stream>>>(A);
      CK(cudaGetLastError(), "deblock launch");
      *n += 2;
    }
    if (p.tools & VVCG_TOOL_SAO)
      for (int c = 0; c < 3; c++, si++) {
        const SaoBoundedPass& S = G.sao_pass[si];
        const uint64_t cnt = (uint64_t)S.w * S.h;
        k_sao_bounded<<<(uint32_t)std::min<uint64_t>((cnt + 255) / 256, (uint64_t)ctx->num_sms * 16), 256, 0,
                        ctx->stream>>>(S);
        CK(cudaGetLastError(), "sao launch");
        (*n)++;
      }
    if (p.tools & VVCG_TOOL_ALF) {
      const AlfGenPass& P = G.alf_pass[ai++];
      const uint64_t nb = (uint64_t)((P.pw + 3) / 4) * ((P.ph + 3) / 4), nc = 2ull * P.cw * P.ch;
      k_alf_general_luma<<<(uint32_t)std::min<uint64_t>((nb + 127) / 128, (uint64_t)ctx->num_sms * 16), 128, 0,
                           ctx->stream>>>(P);
      k_alf_general_chroma<<<(uint32_t)std::min<uint64_t>((nc + 255) / 256, (uint64_t)ctx->num_sms * 16), 256, 0,
                             ctx->stream>>>(P);
      CK(cudaGetLastError(), "alf launch");
      *n += 2;
    }
  }
  return VVCG_OK;
}

}  // namespace

extern "C" {

vvcg_status vvcg_gen_run(vvcg_ctx* ctx, uint32_t graph) {
  if (!ctx) return VVCG_INVALID_INPUT;
  if (!ctx->gen || !ctx->gen->prepared) return fail(ctx, VVCG_INVALID_INPUT, "general batch not prepared");
  GenPass& G = *ctx->gen;
  CK(cudaSetDevice(ctx->device), "cudaSetDevice");
  if (!graph) {
    uint32_t n = 0;
    vvcg_status st = gen_enqueue(ctx, &n);
    ctx->launches += n;
    return st;
  }
  if (!G.exec) {
    CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    uint32_t n = 0;
    vvcg_status st = gen_enqueue(ctx, &n);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
    if (st != VVCG_OK) {
      if (g) cudaGraphDestroy(g);
      return st;
    }
    if (e != cudaSuccess) return cuda_fail(ctx, e, "end capture");
    e = cudaGraphInstantiate(&G.exec, g, 0);
    if (e != cudaSuccess) {
      cudaGraphDestroy(g);
      return cuda_fail(ctx, e, "graph instantiate");
    }
    G.graph = g;
    G.graph_launches = n;
  }
  CK(cudaGraphLaunch(G.exec, ctx->stream), "graph launch");
  ctx->launches += G.graph_launches;
  return VVCG_OK;
}

vvcg_status vvcg_gen_download(vvcg_ctx* ctx, const vvcg_plane_out* out) {
  if (!ctx || !out) return VVCG_INVALID_INPUT;
  if (!ctx->gen || !ctx->gen->prepared) return fail(ctx, VVCG_INVALID_INPUT, "general batch not prepared");
  GenPass& G = *ctx->gen;
  CK(cudaSetDevice(ctx->device), "cudaSetDevice");
  const uint16_t* base = (const uint16_t*)G.planes.p;
  for (size_t i = 0; i < G.pics.size(); i++) {
    const vvcg_gen_pic& p = G.pics[i];
    const GenPicLayout& L = G.lay[i];
    for (int c = 0; c < 3; c++) {
      const vvcg_plane_out& o = out[i * 3 + c];
      if (!o.data) continue;
      const uint32_t w = c ? (p.vis_width + 1) / 2 : p.vis_width, h = c ? (p.vis_height + 1) / 2 : p.vis_height;
      if (o.stride < w) return fail(ctx, VVCG_INVALID_INPUT, "output stride too small");
      CK(cudaMemcpy2DAsync(o.data, (size_t)o.stride * 2, base + L.plane_off[L.final_set][c], (size_t)L.stride[c] * 2,
                           (size_t)w * 2, h, cudaMemcpyDeviceToHost, ctx->stream),
         "download");
    }
  }
  CK(cudaStreamSynchronize(ctx->stream), "download");
  return VVCG_OK;
}

vvcg_status vvcg_decode_general_batch(vvcg_ctx* ctx, const vvcg_gen_batch* b, const vvcg_plane_out* out) {
  vvcg_status st;
  if ((st = vvcg_gen_prepare(ctx, b)) != VVCG_OK) return st;
  if ((st = vvcg_gen_run(ctx, 0)) != VVCG_OK) return st;
  return vvcg_gen_download(ctx, out);
}

}  // extern "C"
