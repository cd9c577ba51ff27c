// mv_api.cu -- host orchestration and the C ABI (include/mvgpu.h).
//
// Replaces the orchestration of Voronoi::build / build_partial (voronoi.rs:151-263):
// dimension normalisation, SimulationBoundary::cuboid, the neighbour structure, the
// per-cell construction, flatten and finalize.  Host-side f64 arithmetic (the
// boundary planes) is compiled without FMA contraction, like the device code.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "../../include/mvgpu.h"
#include "mv_geom.cuh"
#include "mv_internal.h"

namespace mv {
// mv_cells.cu
cudaError_t launch_cells(const Job& J, bool large, int blocks, cudaStream_t st, const JobTable& TB);
size_t cells_big_bytes(int blocks_fast, int blocks_large);
int cells_blocks_per_sm_fast(int precision);
int cells_blocks_per_sm_large(int precision);
// mv_export.cu
void launch_export_count(const int32_t* sid, const int64_t* rec_off, const double* rec, int n,
                         int flags, int64_t* rec_by_orig, int32_t* planes, int32_t* verts,
                         int32_t* tets, int32_t* faces, int32_t* face_verts, cudaStream_t st);
void launch_export_write(const Job& J, const int64_t* rec_by_orig, const double* rec, int n, int flags,
                         const int64_t* plane_off, const int64_t* vert_off, const int64_t* tet_off,
                         const int64_t* face_off, const int64_t* face_vert_base, double* plane_normal,
                         double* plane_point, int32_t* plane_right, uint8_t* plane_code,
                         double* vert_loc, int32_t* vert_dual, double* tet_v, int32_t* tet_plane,
                         int32_t* face_plane, int64_t* face_vert_off, int32_t* face_verts,
                         int64_t n_faces, int64_t n_face_verts, int32_t* status, cudaStream_t st);
// mv_tuning.cu
mv_tuning_entry tuned_params(int dim, int64_t n);
// mv_staged.cu
cudaError_t launch_stage(int kernel, const Job& J, const StageJob& SJ, const JobTable& TB, int blocks,
                         cudaStream_t st);
int stage_blocks_per_sm(int kernel, int precision);
int stage_list_stride();
int stage_wide_stride();
cudaError_t launch_append_range(int32_t* dst, int32_t first, int32_t count, cudaStream_t st);
// cells of the probe chunk that decides between the staged and the fused pipeline
constexpr int64_t STAGE_PROBE_CELLS = 16384;
int64_t stage_record_words(int np, int nv);
// mv_grid.cu
void launch_prep(const double* xyz, int n, int dim, double* gen, unsigned long long* ext_keys,
                 double* ext, int* bad, cudaStream_t st);
void launch_grid_coarse(const double* gen, int n, const int G[3], const double a[3],
                        const double inv[3], int32_t* cid, int32_t* count, int32_t* start,
                        int32_t* dflag, int32_t* dprefix, int dim, long long* scan_tmp, cudaStream_t st);
size_t grid_dense_sort_bytes(int n, int64_t ncell);
void launch_batch_grid(const double* xyz, int n, const int32_t* pos, const int32_t* cbase, int nj,
                       const BatchGrid* bg, int64_t ncell, double* gen, unsigned long long* ext_keys,
                       double* ext, int* bad, int32_t* cid, int32_t* count, int32_t* start,
                       int32_t* dflag, int32_t* dprefix, long long* scan_tmp, cudaStream_t st);
cudaError_t launch_batch_sort(const double* gen, int n, const int32_t* pos, const int32_t* cbase, int nj,
                              const BatchGrid* bg, int64_t ncell, const int32_t* cid, const int32_t* dflag,
                              unsigned long long* key_a, unsigned long long* key_b, int32_t* val_a,
                              int32_t* val_b, void* sort_tmp, size_t sort_bytes, double* sx, double* sy,
                              double* sz, int32_t* sid, uint32_t* fkey, int32_t* start, cudaStream_t st);
void launch_batch_csr(const FaceArrays& f, int64_t F, const int64_t* face_off, const int32_t* face_count,
                      int n, const int32_t* pos, int nj, int32_t* in_count, int32_t* conn_count,
                      cudaStream_t st);
void launch_batch_csr_fill(const FaceArrays& f, int64_t F, const int64_t* face_off, const int64_t* conn_off,
                           const int32_t* in_count, int32_t* cursor, int n, const int32_t* pos, int nj,
                           int32_t* conn, cudaStream_t st);
void launch_batch_localize(FaceArrays& f, int64_t F, const int64_t* face_off, int64_t* conn_off,
                           const int32_t* conn_count, int32_t* conn, int n, const int32_t* pos, int nj,
                           int64_t* fbase, int64_t* cbase_conn, cudaStream_t st);
cudaError_t launch_grid_dense(const double* gen, int n, const int G[3], const double a[3],
                              const double inv[3], int dim, const int32_t* cid, const int32_t* dflag,
                              unsigned long long* key_a, unsigned long long* key_b, int32_t* val_a,
                              int32_t* val_b, void* sort_tmp, size_t sort_bytes, double* sx,
                              double* sy, double* sz, int32_t* sid, uint32_t* fkey, cudaStream_t st);
void launch_scatter(const double* gen, int n, const int32_t* cid, const int32_t* start,
                    int32_t* fill, double* sx, double* sy, double* sz, int32_t* sid, cudaStream_t st);
size_t scan_tmp_elems(int64_t n);
void scan_i32_to_i64(const int32_t* in, int64_t n, int64_t* out, long long* tmp, cudaStream_t st);
void launch_reorder(const FaceArrays& stage, int64_t F, const int64_t* stage_off,
                    const int64_t* face_off, const FaceArrays& out, cudaStream_t st);
void launch_csr_counts(const FaceArrays& f, int64_t F, const int32_t* face_count, int n,
                       int32_t* in_count, int32_t* conn_count, cudaStream_t st);
void launch_csr_fill(const FaceArrays& f, int64_t F, const int64_t* face_off, const int64_t* conn_off,
                     const int32_t* in_count, int32_t* cursor, int n, int32_t* conn, cudaStream_t st);
}  // namespace mv

namespace mv {


// voronoi.rs:200-210 + boundary.rs:14-47 + the grid resolution.
int make_setup(int64_t n, const double* anchor, const double* width, int dim, int periodic,
               const mv_options& o, Setup* s) {
  if (dim < 1 || dim > 3) return MV_ERR_ARG;
  D3 a = {anchor[0], anchor[1], anchor[2]};
  D3 w = {width[0], width[1], width[2]};
  if (dim == 1) {
    a.y = -0.5;
    w.y = 1.0;
  }
  if (dim == 1 || dim == 2) {
    a.z = -0.5;
    w.z = 1.0;
  }
  const double aa[3] = {a.x, a.y, a.z}, ww[3] = {w.x, w.y, w.z};
  for (int i = 0; i < 3; i++) {
    if (!std::isfinite(aa[i]) || !std::isfinite(ww[i]) || !(ww[i] > 0.0)) return MV_ERR_ARG;
    s->anchor[i] = aa[i];
    s->width[i] = ww[i];
  }
  s->dim = dim;
  s->periodic = periodic ? 1 : 0;
  // SimulationBoundary::cuboid
  D3 ba = a, bw = w;
  if (periodic) {
    ba.x -= bw.x;
    bw.x *= 3.0;
    if (dim >= 2) {
      ba.y -= bw.y;
      bw.y *= 3.0;
    }
    if (dim == 3) {
      ba.z -= bw.z;
      bw.z *= 3.0;
    }
  }
  const D3 hi = add(ba, bw);
  const D3 ns[6] = {{1.0, 0.0, 0.0}, {-1.0, 0.0, 0.0}, {0.0, 1.0, 0.0},
                    {0.0, -1.0, 0.0}, {0.0, 0.0, 1.0}, {0.0, 0.0, -1.0}};
  for (int k = 0; k < 6; k++) {
    const D3 p = (k & 1) ? hi : ba;
    s->bn[k][0] = ns[k].x, s->bn[k][1] = ns[k].y, s->bn[k][2] = ns[k].z;
    s->bp[k][0] = p.x, s->bp[k][1] = p.y, s->bp[k][2] = p.z;
    s->bd[k] = dot(ns[k], p);
  }
  const D3 ia = sub(ba, bw);
  s->iloc_a[0] = ia.x, s->iloc_a[1] = ia.y, s->iloc_a[2] = ia.z;
  s->iloc_inv[0] = 1.0 / (3.0 * bw.x);
  s->iloc_inv[1] = 1.0 / (3.0 * bw.y);
  s->iloc_inv[2] = 1.0 / (3.0 * bw.z);
  // parameters the options leave to the library: the tuning table's entry
  const mv_tuning_entry tune = tuned_params(dim, n);
  // uniform grid: ~points_per_grid_cell generators per cell, at most 2^24 cells
  double vol = 1.0;
  for (int i = 0; i < dim; i++) vol *= ww[i];
  const double nn = (double)std::max<int64_t>(n, 1);
  double ppc = o.points_per_grid_cell > 0 ? o.points_per_grid_cell : tune.points_per_grid_cell;
  double h = std::pow(vol * ppc / nn, 1.0 / dim);
  for (;;) {
    int64_t cells = 1;
    for (int i = 0; i < 3; i++) {
      int G = 1;
      if (i < dim) G = (int)std::max(1.0, std::min(std::floor(ww[i] / h), 4096.0));
      s->G[i] = G;
      cells *= G;
    }
    if (cells <= (1ll << 24)) break;
    h *= 1.25;
  }
  for (int i = 0; i < 3; i++) {
    s->gh[i] = ww[i] / s->G[i];
    s->ginv[i] = s->G[i] / ww[i];
    s->geps[i] = 1e-9 * s->gh[i] + 1e-13 * (std::fabs(aa[i]) + ww[i]);
  }
  const double spacing = std::pow(vol / nn, 1.0 / dim);
  const double r0 = o.initial_radius > 0 ? o.initial_radius : tune.initial_radius;
  s->R0 = r0 * spacing;
  return MV_OK;
}

}  // namespace mv

using namespace mv;

namespace {

struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
};

struct Workspace {
  DevBuf in_xyz, in_mask;
  DevBuf gen, sx, sy, sz, sid, cid;
  DevBuf cell_count, cell_start, cell_fill, scan_tmp;
  DevBuf dflag, dprefix, dkey_a, dkey_b, dval_a, dval_b, dsort_tmp, fkey;
  DevBuf volume, centroid, sr, face_count, stage_off, face_off;
  DevBuf in_count, conn_count, conn_off, cursor, conn;
  DevBuf st_left, st_right, st_area, st_cen, st_nrm, st_code;
  DevBuf f_left, f_right, f_area, f_cen, f_nrm, f_code;
  DevBuf ovf_a, ovf_b;
  DevBuf big;  // staging slots of the fused kernel for large shells
  // batches: job table, bases, per-tessellation grids and extents
  DevBuf b_jobs, b_pos, b_cbase, b_grid, b_ext_keys, b_ext, b_fbase, b_cbconn;
  DevBuf counters;
  // staged pipeline: candidate lists, cell records, retry list, per-chunk counters
  DevBuf cand, cand_info, cand_rad, rec_off, rec, retry, retry2, stage_ctr;
  // cell export: record per generator, per-cell sizes and offsets, the CSR arrays
  DevBuf x_rec_by_orig, x_cnt, x_off;
  DevBuf x_pn, x_pp, x_pr, x_pc, x_vl, x_vd, x_tv, x_tp, x_fp, x_fvo, x_fv;
};

}  // namespace

struct mv_context {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev[10] = {};
  int sm_count = 0;
  int bps_fast[2] = {0, 0};
  int bps_large[2] = {0, 0};
  int bps_stage[4][2] = {};  // shell, clip, integral, wide-shell kernels by precision
  std::vector<cudaEvent_t> stage_ev;  // 4 per chunk: before shell, clip, integral, after
  double rec_words_hint = 0.0;  // record words per cell the last staged build needed
  Workspace ws;
  size_t dev_bytes = 0;
  double face_ratio_hint = 0.0;  // faces per cell needed by the last build
  bool large_ran = false;
  bool retry_ran = false;
  mv_build_stats last{};
  // pinned host arena for mv_context_build
  void* host = nullptr;
  size_t host_cap = 0;
  mv_voronoi hv{};
  // host offsets of the last batch build
  std::vector<int64_t> bj_cell, bj_face, bj_conn;
  // pinned host arena for the cells of mv_context_build_cells
  void* host_cells = nullptr;
  size_t host_cells_cap = 0;
  mv_cells hc{};
  // mapped pinned buffer for the build's small device-to-host reads (readback)
  void* rb_host = nullptr;
  void* rb_dev = nullptr;
};

namespace {
constexpr size_t READBACK_BYTES = 1 << 20;

__global__ void readback_kernel(const uint32_t* __restrict__ src, uint32_t* __restrict__ dst, int nwords) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nwords; i += gridDim.x * blockDim.x)
    dst[i] = src[i];
}
}  // namespace

namespace {

int cuda_status(cudaError_t e) {
  if (e == cudaSuccess) return MV_OK;
  if (e == cudaErrorMemoryAllocation) return MV_ERR_OOM;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return MV_ERR_NO_DEVICE;
  return MV_ERR_CUDA;
}

#define MV_CUDA(call)                           \
  do {                                          \
    cudaError_t e_ = (call);                    \
    if (e_ != cudaSuccess) return cuda_status(e_); \
  } while (0)

int ensure(mv_context* ctx, DevBuf& b, size_t bytes) {
  if (bytes == 0) bytes = 16;
  if (b.cap >= bytes) return MV_OK;
  if (b.p) {
    cudaFree(b.p);
    ctx->dev_bytes -= b.cap;
    b.p = nullptr;
    b.cap = 0;
  }
  size_t want = bytes + bytes / 8;  // headroom for slightly larger rebuilds
  cudaError_t e = cudaMalloc(&b.p, want);
  if (e != cudaSuccess) {
    cudaGetLastError();
    e = cudaMalloc(&b.p, bytes);
    want = bytes;
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    b.p = nullptr;
    return MV_ERR_OOM;
  }
  b.cap = want;
  ctx->dev_bytes += want;
  return MV_OK;
}

template <class T>
T* P(DevBuf& b) {
  return static_cast<T*>(b.p);
}

// A small device-to-host read inside a build (counters, sizes), complete on return.
// It goes through a kernel into the context's mapped pinned buffer rather than a
// cudaMemcpy: a copy would queue on the copy engine behind any bulk result copy that
// another context has in flight, stalling this build until that copy ends.
int readback(mv_context* ctx, void* dst, const void* src, size_t bytes, cudaStream_t st) {
  if (bytes == 0) return MV_OK;
  if (ctx->rb_dev && bytes % 4 == 0 && bytes <= READBACK_BYTES &&
      reinterpret_cast<uintptr_t>(src) % 4 == 0) {
    const int nw = (int)(bytes / 4);
    readback_kernel<<<std::min(64, (nw + 255) / 256), 256, 0, st>>>(
        static_cast<const uint32_t*>(src), static_cast<uint32_t*>(ctx->rb_dev), nw);
    MV_CUDA(cudaGetLastError());
    MV_CUDA(cudaStreamSynchronize(st));
    std::memcpy(dst, ctx->rb_host, bytes);
    return MV_OK;
  }
  MV_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st));
  MV_CUDA(cudaStreamSynchronize(st));
  return MV_OK;
}

#define MV_RB(dst, src, bytes)                            \
  do {                                                    \
    const int rb_ = readback(ctx, (dst), (src), (bytes), st); \
    if (rb_) return rb_;                                  \
  } while (0)

double face_ratio(int dim, int face_mode) {
  if (dim == 3) return face_mode == MV_FACES_ALL ? 17.5 : 10.5;
  if (dim == 2) return face_mode == MV_FACES_ALL ? 7.5 : 4.5;
  return 2.5;
}

// The automatic pipeline is the tuning table's for the build's band (staged for builds
// large enough to fill the GPU with chunks); the candidate list packs a sorted
// position with a shift code into 32 bits.
bool use_staged(const mv_options& o, int64_t n, int dim) {
  if (n <= 0 || n >= (int64_t)(0xffffffffu / 27u)) return false;
  if (o.pipeline == MV_PIPELINE_STAGED) return true;
  if (o.pipeline == MV_PIPELINE_FUSED) return false;
  return tuned_params(dim, n).pipeline == MV_PIPELINE_STAGED;
}

int64_t record_words_per_cell(int dim) { return dim == 3 ? 352 : (dim == 2 ? 224 : 128); }

// Shell, clip and integral kernels over chunks of cells in processing (grid) order.
// Cells the first shell does not decide are appended to the retry list; *n_retry
// receives their number.
int run_staged(mv_context* ctx, const Job& J, const JobTable& TB, int dim, const mv_options& o,
               int64_t n, int pi, cudaStream_t st, int64_t* launches, int64_t* n_retry,
               double ms_stage[3], unsigned long long* keep_records, int64_t* n_wide,
               const int32_t** retry_order) {
  Workspace& W = ctx->ws;
  // an export build keeps every cell's record: one chunk, and the record counter the
  // fused kernel shares (keep_records)
  const int64_t chunk = keep_records ? n
                                     : std::min<int64_t>(n, o.chunk_cells > 0 ? o.chunk_cells
                                                                              : tuned_params(dim, n).chunk_cells);
  // chunks (first item, items); with the automatic pipeline a small probe chunk comes
  // first: when most of its cells need the exact predicate (an exact lattice: every
  // vertex is shared by co-spherical generators) the staged kernels would only hand
  // the remaining cells on as well, so they go to the fused kernel directly
  const bool probe = !keep_records && o.pipeline == MV_PIPELINE_AUTO && n >= 4 * STAGE_PROBE_CELLS &&
                     chunk > STAGE_PROBE_CELLS;
  std::vector<std::pair<int64_t, int64_t>> chunks;
  for (int64_t p0 = 0; p0 < n;) {
    const int64_t m = (probe && p0 == 0) ? STAGE_PROBE_CELLS : std::min<int64_t>(chunk, n - p0);
    chunks.push_back({p0, m});
    p0 += m;
  }
  const int64_t nchunks = (int64_t)chunks.size();
  const int stride = stage_list_stride();
  int64_t wpc = std::max<int64_t>(record_words_per_cell(dim), (int64_t)ctx->rec_words_hint);
  wpc = std::min<int64_t>(wpc, stage_record_words(64, 64));
  const int64_t rec_cap = chunk * wpc;
  // the wide round re-chunks the retry list so that its longer lists fit the same
  // candidate buffer
  const int wstride = stage_wide_stride();
  const int64_t chunk2 = std::max<int64_t>(1, chunk * stride / wstride);
  const int64_t nchunks2 = (n + chunk2 - 1) / chunk2;
  const size_t ctr2 = 1 + 3 * (size_t)nchunks;  // wide-round words start here
  const size_t ctr_words = ctr2 + 1 + 3 * (size_t)nchunks2;
  int e = 0;
  e |= ensure(ctx, W.cand, 4 * (size_t)chunk * stride);
  e |= ensure(ctx, W.cand_info, 4 * (size_t)chunk);
  e |= ensure(ctx, W.cand_rad, 8 * (size_t)chunk);
  e |= ensure(ctx, W.rec_off, 8 * (size_t)chunk);
  e |= ensure(ctx, W.rec, 8 * (size_t)rec_cap);
  e |= ensure(ctx, W.retry, 4 * (size_t)n);
  if (!keep_records) e |= ensure(ctx, W.retry2, 4 * (size_t)n);
  e |= ensure(ctx, W.stage_ctr, 8 * ctr_words);
  if (e) return MV_ERR_OOM;
  unsigned long long* ctr = P<unsigned long long>(W.stage_ctr);
  MV_CUDA(cudaMemsetAsync(ctr, 0, 8 * ctr_words, st));
  while (ctx->stage_ev.size() < 4 * (size_t)std::max(nchunks, nchunks2)) {
    cudaEvent_t ev;
    MV_CUDA(cudaEventCreate(&ev));
    ctx->stage_ev.push_back(ev);
  }
  StageJob SJ;
  std::memset(&SJ, 0, sizeof(SJ));
  SJ.cstride = stride;
  SJ.cand = P<uint32_t>(W.cand);
  SJ.info = P<int32_t>(W.cand_info);
  SJ.rad = P<double>(W.cand_rad);
  SJ.rec_off = P<int64_t>(W.rec_off);
  SJ.rec = P<double>(W.rec);
  SJ.rec_cap = rec_cap;
  SJ.full_records = keep_records ? 1 : 0;
  // box-corner band tests (quantised lattices) are decided by the clip kernel's box
  // form, in the probe chunk and, when the probe met them in every cell on average,
  // in every later chunk
  bool box_mode = false;
  SJ.retry_list = P<int32_t>(W.retry);
  SJ.retry_count = reinterpret_cast<unsigned int*>(ctr);
  // cells that need the exact predicate skip the wide round: they join the list the
  // fused kernel takes (the wide round's retry list; with kept records, the one list)
  SJ.fused_list = keep_records ? SJ.retry_list : P<int32_t>(W.retry2);
  SJ.fused_count = keep_records ? SJ.retry_count : reinterpret_cast<unsigned int*>(ctr + ctr2);
  for (int64_t c = 0; c < nchunks; c++) {
    SJ.item0 = (int32_t)chunks[c].first;
    SJ.nitems = (int32_t)chunks[c].second;
    SJ.work = reinterpret_cast<unsigned int*>(ctr + 1 + 3 * c);
    SJ.rec_counter = keep_records ? keep_records : ctr + 1 + 3 * c + 2;
    SJ.box = ((probe && c == 0) || box_mode) ? 1 : 0;
    const int64_t warps_needed = SJ.nitems;
    for (int k = 0; k < 3; k++) {
      const int wpb = 4;  // every stage kernel runs 4 warps per block
      int64_t blocks = (int64_t)ctx->sm_count * std::max(1, ctx->bps_stage[k][pi]);
      blocks = std::min<int64_t>(blocks, (warps_needed + wpb - 1) / wpb);
      MV_CUDA(cudaEventRecord(ctx->stage_ev[4 * c + k], st));
      MV_CUDA(launch_stage(k, J, SJ, TB, (int)std::max<int64_t>(1, blocks), st));
      (*launches)++;
    }
    MV_CUDA(cudaEventRecord(ctx->stage_ev[4 * c + 3], st));
    if (probe && c == 0) {
      unsigned long long pc[3] = {0, 0, 0};
      MV_RB(&pc[0], ctr, 8);
      MV_RB(&pc[1], ctr + ctr2, 8);
      MV_RB(&pc[2], J.stats + ST_EXACT, 8);
      const int64_t n_exact = (int64_t)(pc[1] & 0xffffffffull);
      box_mode = (int64_t)pc[2] >= (int64_t)SJ.nitems;
      if (2 * n_exact >= SJ.nitems) {
        // the fused kernel's list: the probe's exact cells, its retries, then every
        // cell after the probe
        const int64_t n_ret = (int64_t)(pc[0] & 0xffffffffull);
        int32_t* fl = P<int32_t>(W.retry2);
        if (n_ret > 0)
          MV_CUDA(cudaMemcpyAsync(fl + n_exact, P<int32_t>(W.retry), 4 * (size_t)n_ret,
                                  cudaMemcpyDeviceToDevice, st));
        MV_CUDA(launch_append_range(fl + n_exact + n_ret, (int32_t)SJ.nitems, (int32_t)(n - SJ.nitems), st));
        (*launches)++;
        for (int k = 0; k < 3; k++) {
          float t = 0.f;
          cudaEventElapsedTime(&t, ctx->stage_ev[k], ctx->stage_ev[k + 1]);
          ms_stage[k] = t;
        }
        *n_retry = n_exact + n_ret + (n - SJ.nitems);
        *n_wide = 0;
        *retry_order = fl;
        return MV_OK;
      }
    }
  }
  std::vector<unsigned long long> h(ctr_words);
  MV_RB(h.data(), ctr, 8 * (ctr2 + 1));
  // the first round's retries: for the wide round, or with kept records (one list,
  // exact cells included) for the fused kernel
  const int64_t n_first = (int64_t)(h[0] & 0xffffffffull);
  *n_retry = n_first;
  *n_wide = 0;
  *retry_order = P<int32_t>(W.retry);
  if (!keep_records) {
    // the fused kernel's list so far: the cells that needed the exact predicate
    *retry_order = P<int32_t>(W.retry2);
    *n_retry = (int64_t)(h[ctr2] & 0xffffffffull);
  }
  for (int k = 0; k < 3; k++) ms_stage[k] = 0.0;
  for (int64_t c = 0; c < nchunks; c++) {
    for (int k = 0; k < 3; k++) {
      float t = 0.f;
      cudaEventElapsedTime(&t, ctx->stage_ev[4 * c + k], ctx->stage_ev[4 * c + k + 1]);
      ms_stage[k] += t;
    }
  }
  if (!keep_records && n_first > 0) {
    // the wide round over the retry list; what it cannot close goes to the fused kernel
    const int64_t nr = n_first;
    StageJob SW = SJ;
    SW.cstride = wstride;
    SW.order = P<int32_t>(W.retry);
    SW.retry_list = P<int32_t>(W.retry2);
    SW.retry_count = reinterpret_cast<unsigned int*>(ctr + ctr2);
    SW.fused_list = SW.retry_list;
    SW.fused_count = SW.retry_count;
    const int64_t nc = (nr + chunk2 - 1) / chunk2;
    for (int64_t c = 0; c < nc; c++) {
      SW.item0 = (int32_t)(c * chunk2);
      SW.nitems = (int32_t)std::min<int64_t>(chunk2, nr - c * chunk2);
      SW.work = reinterpret_cast<unsigned int*>(ctr + ctr2 + 1 + 3 * c);
      SW.rec_counter = ctr + ctr2 + 1 + 3 * c + 2;
      const int kern[3] = {3, 1, 2};
      for (int k = 0; k < 3; k++) {
        int64_t blocks = (int64_t)ctx->sm_count * std::max(1, ctx->bps_stage[kern[k]][pi]);
        blocks = std::min<int64_t>(blocks, (SW.nitems + 3) / 4);
        MV_CUDA(cudaEventRecord(ctx->stage_ev[4 * c + k], st));
        MV_CUDA(launch_stage(kern[k], J, SW, TB, (int)std::max<int64_t>(1, blocks), st));
        (*launches)++;
      }
      MV_CUDA(cudaEventRecord(ctx->stage_ev[4 * c + 3], st));
    }
    unsigned long long r2 = 0;
    MV_RB(&r2, ctr + ctr2, 8);
    for (int64_t c = 0; c < nc; c++) {
      for (int k = 0; k < 3; k++) {
        float t = 0.f;
        cudaEventElapsedTime(&t, ctx->stage_ev[4 * c + k], ctx->stage_ev[4 * c + k + 1]);
        ms_stage[k] += t;
      }
    }
    *n_wide = nr;
    *n_retry = (int64_t)(r2 & 0xffffffffull);
    *retry_order = P<int32_t>(W.retry2);
  }
  // size the record buffer of the next build by what this one asked for
  double need = 0.0;
  for (int64_t c = 0; c < nchunks; c++) {
    const int64_t items = chunks[c].second;
    need = std::max(need, (double)h[1 + 3 * c + 2] / (double)std::max<int64_t>(items, 1));
  }
  if (!keep_records && need * 1.1 > (double)wpc) ctx->rec_words_hint = need * 1.2;
  return MV_OK;
}

// Fast-tier grid of the fused kernel for `cells` cells: the resident maximum, or fewer
// blocks for small counts (at least four cells per warp, so that a small build's
// warps, and their staging slots, stay few).
int fused_blocks(const mv_context* ctx, int pi, int64_t cells) {
  const int64_t full = (int64_t)ctx->sm_count * std::max(1, ctx->bps_fast[pi]);
  return (int)std::max<int64_t>(1, std::min<int64_t>(full, (cells + 15) / 16));
}

// The tessellation-specific geometry of a Job: its grid, boundary planes (boundary.rs:
// 14-47), iloc frame (boundary.rs:49-64), periodic image offsets (rtree_nn.rs:27-33,
// 86), first shell radius and Morton key width.
void set_job_geometry(Job& J, const Setup& s) {
  for (int i = 0; i < 3; i++) {
    J.G[i] = s.G[i];
    J.ga[i] = s.anchor[i];
    J.gw[i] = s.width[i];
    J.gh[i] = s.gh[i];
    J.ginv[i] = s.ginv[i];
    J.geps[i] = s.geps[i];
    J.iloc_a[i] = s.iloc_a[i];
    J.iloc_inv[i] = s.iloc_inv[i];
  }
  J.dim = s.dim;
  J.periodic = s.periodic;
  J.R0 = s.R0;
  J.fbits = fkey_bits(s.dim);
  for (int c = 0; c < 27; c++) {
    const int m[3] = {c % 3 - 1, (c / 3) % 3 - 1, c / 9 - 1};
    for (int i = 0; i < 3; i++) {
      const double q = (double)(-m[i]) * s.width[i];
      J.qshift[c][i] = q;
      J.shift[c][i] = -q;
    }
  }
  for (int k = 0; k < 6; k++) {
    for (int i = 0; i < 3; i++) J.bn[k][i] = s.bn[k][i], J.bp[k][i] = s.bp[k][i];
    J.bd[k] = s.bd[k];
  }
}

// Staging-slot bytes of the fused kernel for a build of n cells: one slot per warp of
// the largest fast-tier or large-tier grid the build can launch (fused_blocks; a
// large-tier grid has at most one block per cell).
size_t big_slot_bytes(const mv_context* ctx, int pi, int64_t n) {
  const int64_t sm = ctx->sm_count;
  const int64_t fast = fused_blocks(ctx, pi, n);
  const int64_t large = std::min<int64_t>(sm * std::max(1, ctx->bps_large[pi]), n);
  return cells_big_bytes((int)std::max<int64_t>(fast, 1), (int)std::max<int64_t>(large, 1));
}

// The cell phase of a build, after the grid: the staged rounds (or the fused kernel
// alone), the fused kernel on what they left, the large tier on the cells that outgrew
// the fast one; reads the device counters back into *hc.  J is the build's Job (for a
// batch, the template Job whose shared fields all tessellations use; TB its job table).
int run_cell_phase(mv_context* ctx, const Job& J, const JobTable& TB, int dim, const mv_options& o,
                   int64_t n, int pi, bool staged, bool exporting, cudaStream_t st, int64_t* launches,
                   mv_build_stats* stats, DevCounters* hc) {
  Workspace& W = ctx->ws;
  DevCounters* C = P<DevCounters>(W.counters);
  bool retry_ran = false;
  int64_t n_retry = 0, n_wide = 0;
  double ms_stage[3] = {0.0, 0.0, 0.0};
  MV_CUDA(cudaEventRecord(ctx->ev[1], st));
  if (n > 0 && staged) {
    const int32_t* retry_order = nullptr;
    int rc2 = run_staged(ctx, J, TB, dim, o, n, pi, st, launches, &n_retry, ms_stage,
                         exporting ? &C->rec_counter : nullptr, &n_wide, &retry_order);
    if (rc2) return rc2;
    MV_CUDA(cudaEventRecord(ctx->ev[2], st));
    if (n_retry > 0) {
      // cells neither staged round closed: the fused kernel builds them
      Job Rj = J;
      Rj.order = retry_order;
      Rj.n_order = (int32_t)n_retry;
      // one warp per cell, within the grid the slots were sized for
      const int blocks = (int)std::min<int64_t>(fused_blocks(ctx, pi, n), (n_retry + 3) / 4);
      MV_CUDA(cudaEventRecord(ctx->ev[7], st));
      MV_CUDA(launch_cells(Rj, false, blocks, st, TB));
      MV_CUDA(cudaEventRecord(ctx->ev[8], st));
      (*launches)++;
      retry_ran = true;
    }
  } else {
    if (n > 0) {
      MV_CUDA(launch_cells(J, false, fused_blocks(ctx, pi, n), st, TB));
      (*launches)++;
    }
    MV_CUDA(cudaEventRecord(ctx->ev[2], st));
  }
  ctx->retry_ran = retry_ran;
  stats->staged_retries = n_retry;
  stats->staged_wide = n_wide;
  stats->ms_shell = ms_stage[0];
  stats->ms_clip = ms_stage[1];
  stats->ms_integrate = ms_stage[2];
  bool large_ran = false;
  MV_RB(hc, C, sizeof(DevCounters));
  if (hc->bad_input) return MV_ERR_ARG;
  const unsigned novf = hc->ovf_count[0];
  if (novf > 0 && !hc->status[STATUS_CODE]) {
    // cells that outgrew the fast tier: the large tier rebuilds them
    Job L = J;
    L.order = P<int32_t>(W.ovf_a);
    L.n_order = (int32_t)novf;
    L.work_counter = &C->work[1];
    L.ovf_list = P<int32_t>(W.ovf_b);
    L.ovf_count = &C->ovf_count[1];
    int blocks = ctx->sm_count * std::max(1, ctx->bps_large[pi]);
    blocks = std::min<int>(blocks, (int)novf);
    MV_CUDA(cudaEventRecord(ctx->ev[3], st));
    MV_CUDA(launch_cells(L, true, blocks, st, TB));
    MV_CUDA(cudaEventRecord(ctx->ev[4], st));
    (*launches)++;
    large_ran = true;
    MV_RB(hc, C, sizeof(DevCounters));
  }
  ctx->large_ran = large_ran;
  return MV_OK;
}

// Cells export (mv_export.cu): records by generator, sizes, offsets, then the arrays.
int export_cells(mv_context* ctx, const Job& J, int64_t n, int flags, cudaStream_t st,
                 int64_t* launches, mv_cells* out) {
  Workspace& W = ctx->ws;
  const size_t N = (size_t)std::max<int64_t>(n, 1);
  int e = 0;
  e |= ensure(ctx, W.x_rec_by_orig, 8 * N);
  e |= ensure(ctx, W.x_cnt, 4 * 5 * N);
  e |= ensure(ctx, W.x_off, 8 * 5 * (N + 1));
  if (e) return MV_ERR_OOM;
  int32_t* cnt = P<int32_t>(W.x_cnt);
  int64_t* off = P<int64_t>(W.x_off);
  const int ni = (int)n;
  launch_export_count(J.sid, J.rec_off, J.rec, ni, flags, P<int64_t>(W.x_rec_by_orig), cnt,
                      cnt + N, cnt + 2 * N, cnt + 3 * N, cnt + 4 * N, st);
  (*launches)++;
  int64_t tot[5] = {0, 0, 0, 0, 0};
  if (n > 0) {
    for (int k = 0; k < 5; k++) {
      scan_i32_to_i64(cnt + k * N, n, off + k * (N + 1), P<long long>(W.scan_tmp), st);
      MV_RB(&tot[k], off + k * (N + 1) + n, 8);
    }
    *launches += 15;
  } else {
    MV_CUDA(cudaMemsetAsync(off, 0, 8 * 5 * (N + 1), st));
  }
  MV_CUDA(cudaStreamSynchronize(st));
  const size_t P_ = (size_t)std::max<int64_t>(tot[0], 1), V = (size_t)std::max<int64_t>(tot[1], 1),
               T = (size_t)std::max<int64_t>(tot[2], 1), Fc = (size_t)std::max<int64_t>(tot[3], 1),
               FV = (size_t)std::max<int64_t>(tot[4], 1);
  e = 0;
  e |= ensure(ctx, W.x_pn, 24 * P_);
  e |= ensure(ctx, W.x_pp, 24 * P_);
  e |= ensure(ctx, W.x_pr, 4 * P_);
  e |= ensure(ctx, W.x_pc, P_);
  e |= ensure(ctx, W.x_vl, 24 * V);
  e |= ensure(ctx, W.x_vd, 12 * V);
  if (flags & MV_CELLS_TETS) e |= ensure(ctx, W.x_tv, 72 * T) | ensure(ctx, W.x_tp, 4 * T);
  if (flags & MV_CELLS_WITH_FACES)
    e |= ensure(ctx, W.x_fp, 4 * Fc) | ensure(ctx, W.x_fvo, 8 * (Fc + 1)) | ensure(ctx, W.x_fv, 4 * FV);
  if (e) return MV_ERR_OOM;
  DevCounters* C = P<DevCounters>(W.counters);
  launch_export_write(J, P<int64_t>(W.x_rec_by_orig), J.rec, ni, flags, off, off + (N + 1),
                      off + 2 * (N + 1), off + 3 * (N + 1), off + 4 * (N + 1), P<double>(W.x_pn),
                      P<double>(W.x_pp), P<int32_t>(W.x_pr), P<uint8_t>(W.x_pc), P<double>(W.x_vl),
                      P<int32_t>(W.x_vd), P<double>(W.x_tv), P<int32_t>(W.x_tp), P<int32_t>(W.x_fp),
                      P<int64_t>(W.x_fvo), P<int32_t>(W.x_fv), tot[3], tot[4], C->status, st);
  *launches += (flags & MV_CELLS_WITH_FACES) ? 2 : 1;
  MV_CUDA(cudaGetLastError());
  int32_t status[STATUS_WORDS];
  MV_RB(status, C->status, sizeof(status));
  if (status[STATUS_CODE]) return status[STATUS_CODE];
  std::memset(out, 0, sizeof(*out));
  out->n_cells = n;
  out->n_planes = tot[0], out->n_vertices = tot[1];
  out->n_tets = (flags & MV_CELLS_TETS) ? tot[2] : 0;
  out->n_faces = (flags & MV_CELLS_WITH_FACES) ? tot[3] : 0;
  out->n_face_vertices = (flags & MV_CELLS_WITH_FACES) ? tot[4] : 0;
  out->cell_plane_offset = off;
  out->plane_normal = P<double>(W.x_pn);
  out->plane_point = P<double>(W.x_pp);
  out->plane_right = P<int32_t>(W.x_pr);
  out->plane_shift_code = P<uint8_t>(W.x_pc);
  out->cell_vertex_offset = off + (N + 1);
  out->vertex_loc = P<double>(W.x_vl);
  out->vertex_dual = P<int32_t>(W.x_vd);
  if (flags & MV_CELLS_TETS) {
    out->cell_tet_offset = off + 2 * (N + 1);
    out->tet_vertices = P<double>(W.x_tv);
    out->tet_plane = P<int32_t>(W.x_tp);
  }
  if (flags & MV_CELLS_WITH_FACES) {
    out->cell_face_offset = off + 3 * (N + 1);
    out->face_plane = P<int32_t>(W.x_fp);
    out->face_vertex_offset = P<int64_t>(W.x_fvo);
    out->face_vertices = P<int32_t>(W.x_fv);
  }
  return MV_OK;
}

int build_device_impl(mv_context* ctx, const double* d_xyz, const uint8_t* d_mask, int64_t n,
                      const double* anchor, const double* width, int dim, int periodic,
                      const mv_options* opts_in, mv_device_voronoi* out, int cells_flags = -1,
                      mv_cells* cells_out = nullptr) {
  mv_options o;
  mv_options_default(&o);
  if (opts_in) o = *opts_in;
  if (!out || n < 0 || (n > 0 && !d_xyz)) return MV_ERR_ARG;
  if (n >= (int64_t)(0xffffffffu / 27u)) return MV_ERR_ARG;  // neighbour tie key range
  if (o.precision != MV_PRECISION_FP64 && o.precision != MV_PRECISION_FILTERED) return MV_ERR_ARG;
  if (o.face_mode != MV_FACES_OWNED && o.face_mode != MV_FACES_ALL) return MV_ERR_ARG;
  if (o.pipeline < MV_PIPELINE_AUTO || o.pipeline > MV_PIPELINE_FUSED || o.chunk_cells < 0)
    return MV_ERR_ARG;
  const bool exporting = cells_flags >= 0;
  if (exporting && (!cells_out || (cells_flags & ~(MV_CELLS_TETS | MV_CELLS_WITH_FACES))))
    return MV_ERR_ARG;
  if (exporting && (cells_flags & MV_CELLS_WITH_FACES) && dim != 3) return MV_ERR_ARG;  // with_faces: 3D
  Setup s;
  int rc = make_setup(n, anchor, width, dim, periodic, o, &s);
  if (rc) return rc;
  MV_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t st = o.stream ? (cudaStream_t)o.stream : ctx->stream;
  Workspace& W = ctx->ws;
  const int ni = (int)n;
  const int64_t ncell = (int64_t)s.G[0] * s.G[1] * s.G[2];
  const size_t N = (size_t)std::max<int64_t>(n, 1);

  // ---- workspace ----
  int e = 0;
  e |= ensure(ctx, W.gen, 24 * N);
  e |= ensure(ctx, W.sx, 8 * N);
  e |= ensure(ctx, W.sy, 8 * N);
  e |= ensure(ctx, W.sz, 8 * N);
  e |= ensure(ctx, W.sid, 4 * N);
  e |= ensure(ctx, W.cid, 4 * N);
  e |= ensure(ctx, W.cell_count, 4 * (ncell + 1));
  e |= ensure(ctx, W.cell_start, 4 * (ncell + 1));
  e |= ensure(ctx, W.cell_fill, 4 * (ncell + 1));
  e |= ensure(ctx, W.dflag, 4 * (ncell + 1));
  e |= ensure(ctx, W.dprefix, 4 * (ncell + 1));
  e |= ensure(ctx, W.scan_tmp, 8 * (scan_tmp_elems(std::max<int64_t>(ncell + 1, N)) + 64));
  e |= ensure(ctx, W.volume, 8 * N);
  e |= ensure(ctx, W.centroid, 24 * N);
  e |= ensure(ctx, W.sr, 8 * N);
  e |= ensure(ctx, W.face_count, 4 * N);
  e |= ensure(ctx, W.stage_off, 8 * N);
  e |= ensure(ctx, W.face_off, 8 * (N + 1));
  e |= ensure(ctx, W.in_count, 4 * N);
  e |= ensure(ctx, W.conn_count, 4 * N);
  e |= ensure(ctx, W.conn_off, 8 * (N + 1));
  e |= ensure(ctx, W.cursor, 4 * N);
  e |= ensure(ctx, W.ovf_a, 4 * N);
  e |= ensure(ctx, W.ovf_b, 4 * N);
  e |= ensure(ctx, W.counters, sizeof(DevCounters));
  if (e) return MV_ERR_OOM;
  double ratio = std::max(face_ratio(s.dim, o.face_mode), ctx->face_ratio_hint);
  int64_t face_cap = (int64_t)(ratio * (double)n) + 4096;

  DevCounters* C = P<DevCounters>(W.counters);
  mv_build_stats stats{};
  int64_t launches = 0;
  int64_t F = 0;
  for (int attempt = 0;; attempt++) {
    size_t FC = (size_t)face_cap;
    e = 0;
    e |= ensure(ctx, W.st_left, 4 * FC);
    e |= ensure(ctx, W.st_right, 4 * FC);
    e |= ensure(ctx, W.st_area, 8 * FC);
    e |= ensure(ctx, W.st_cen, 24 * FC);
    e |= ensure(ctx, W.st_nrm, 24 * FC);
    e |= ensure(ctx, W.st_code, FC);
    if (e) return MV_ERR_OOM;
    face_cap = (int64_t)std::min(W.st_left.cap / 4, W.st_code.cap);
    face_cap = std::min<int64_t>(face_cap, (int64_t)(W.st_area.cap / 8));
    face_cap = std::min<int64_t>(face_cap, (int64_t)(W.st_cen.cap / 24));

    // ---- clear counters ----
    MV_CUDA(cudaMemsetAsync(C, 0, sizeof(DevCounters), st));
    // the failing cell is a minimum over the failing cells: start above every index
    MV_CUDA(cudaMemsetAsync(C->status + STATUS_CELL, 0x7f, sizeof(int32_t), st));
    MV_CUDA(cudaMemsetAsync(C->ext_keys, 0xff, 3 * sizeof(unsigned long long), st));
    MV_CUDA(cudaMemsetAsync(W.cell_count.p, 0, 4 * (ncell + 1), st));
    MV_CUDA(cudaMemsetAsync(W.cell_fill.p, 0, 4 * (ncell + 1), st));

    // ---- generators + grid (replaces build_rtree, rtree_nn.rs:6-8) ----
    MV_CUDA(cudaEventRecord(ctx->ev[0], st));
    launches = 13;  // prep, extent, cell index, 3 x 3 scan kernels, dense flags, scatter
    launch_prep(d_xyz, ni, s.dim, P<double>(W.gen), C->ext_keys, C->ext, &C->bad_input, st);
    launch_grid_coarse(P<double>(W.gen), ni, s.G, s.anchor, s.ginv, P<int32_t>(W.cid),
                       P<int32_t>(W.cell_count), P<int32_t>(W.cell_start), P<int32_t>(W.dflag),
                       P<int32_t>(W.dprefix), s.dim, P<long long>(W.scan_tmp), st);
    int32_t ndense = 0;
    MV_RB(&ndense, P<int32_t>(W.dprefix) + ncell, 4);
    if (ndense > 0) {
      // clustered input: the dense cells are ordered by Morton key (a radix sort)
      const size_t sort_bytes = grid_dense_sort_bytes(ni, ncell);
      e = 0;
      e |= ensure(ctx, W.dkey_a, 8 * N);
      e |= ensure(ctx, W.dkey_b, 8 * N);
      e |= ensure(ctx, W.dval_a, 4 * N);
      e |= ensure(ctx, W.dval_b, 4 * N);
      e |= ensure(ctx, W.fkey, 4 * N);
      e |= ensure(ctx, W.dsort_tmp, sort_bytes + 256);
      if (e) return MV_ERR_OOM;
      MV_CUDA(launch_grid_dense(P<double>(W.gen), ni, s.G, s.anchor, s.ginv, s.dim, P<int32_t>(W.cid),
                                P<int32_t>(W.dflag), P<unsigned long long>(W.dkey_a),
                                P<unsigned long long>(W.dkey_b), P<int32_t>(W.dval_a),
                                P<int32_t>(W.dval_b), W.dsort_tmp.p, W.dsort_tmp.cap, P<double>(W.sx),
                                P<double>(W.sy), P<double>(W.sz), P<int32_t>(W.sid),
                                P<uint32_t>(W.fkey), st));
      launches += 6;  // keys, gather and the sort's passes
    } else {
      launch_scatter(P<double>(W.gen), ni, P<int32_t>(W.cid), P<int32_t>(W.cell_start),
                     P<int32_t>(W.cell_fill), P<double>(W.sx), P<double>(W.sy), P<double>(W.sz),
                     P<int32_t>(W.sid), st);
    }

    // ---- cells ----
    Job J;
    std::memset(&J, 0, sizeof(J));
    J.gen = P<double>(W.gen);
    J.sx = P<double>(W.sx);
    J.sy = P<double>(W.sy);
    J.sz = P<double>(W.sz);
    J.sid = P<int32_t>(W.sid);
    J.cell_start = P<int32_t>(W.cell_start);
    if (ndense > 0) {
      J.dprefix = P<int32_t>(W.dprefix);
      J.cell_dense = P<int32_t>(W.dflag);
      J.fkey = P<uint32_t>(W.fkey);
    }
    J.mask = d_mask;
    J.n = ni;
    J.face_mode = o.face_mode;
    J.precision = o.precision;
    set_job_geometry(J, s);
    J.ext = C->ext;
    J.ppc_mean = (double)std::max<int64_t>(n, 1) / (double)ncell;
    J.volume = P<double>(W.volume);
    J.centroid = P<double>(W.centroid);
    J.safety_radius = P<double>(W.sr);
    J.face_count = P<int32_t>(W.face_count);
    J.stage_off = P<int64_t>(W.stage_off);
    J.f_left = P<int32_t>(W.st_left);
    J.f_right = P<int32_t>(W.st_right);
    J.f_area = P<double>(W.st_area);
    J.f_centroid = P<double>(W.st_cen);
    J.f_normal = P<double>(W.st_nrm);
    J.f_code = P<uint8_t>(W.st_code);
    J.face_counter = &C->face_counter;
    J.face_cap = face_cap;
    J.order = nullptr;
    J.n_order = ni;
    J.work_counter = &C->work[0];
    J.ovf_list = P<int32_t>(W.ovf_a);
    J.ovf_count = &C->ovf_count[0];
    J.status = C->status;
    J.stats = C->stats;
    const int pi = o.precision == MV_PRECISION_FILTERED ? 1 : 0;
    {
      if (ensure(ctx, W.big, big_slot_bytes(ctx, pi, n))) return MV_ERR_OOM;
      J.big = static_cast<char*>(W.big.p);
    }
    const bool staged = use_staged(o, n, s.dim);
    if (exporting) {
      // every built cell leaves a record: the staged clip kernel and the fused kernel
      // (retries, small builds, the large tier) write them to one buffer
      int64_t wpc = std::max<int64_t>(record_words_per_cell(s.dim), (int64_t)ctx->rec_words_hint);
      const int64_t cap = (int64_t)N * wpc;
      if (ensure(ctx, W.rec_off, 8 * N) || ensure(ctx, W.rec, 8 * (size_t)cap)) return MV_ERR_OOM;
      MV_CUDA(cudaMemsetAsync(W.rec_off.p, 0xff, 8 * N, st));
      J.rec = P<double>(W.rec);
      J.rec_cap = (int64_t)(W.rec.cap / 8);
      J.rec_counter = &C->rec_counter;
      J.rec_off = P<int64_t>(W.rec_off);
    }
    DevCounters hc;
    {
      const int rcp = run_cell_phase(ctx, J, JobTable{nullptr, nullptr, 0}, s.dim, o, n, pi, staged,
                                     exporting, st, &launches, &stats, &hc);
      if (rcp) return rcp;
    }
    if (hc.status[STATUS_CODE]) {
      std::memset(out, 0, sizeof(*out));
      out->n_cells = n;
      out->error_cell = hc.status[STATUS_CELL];
      return hc.status[STATUS_CODE];
    }
    if (hc.ovf_count[1] > 0) return MV_ERR_CAPACITY;
    if (hc.status[STATUS_REC_OVERFLOW]) {
      // the cell records did not fit: size the buffer from what was asked, rerun
      if (attempt >= 2) return MV_ERR_CAPACITY;
      ctx->rec_words_hint = 1.2 * (double)hc.rec_counter / (double)std::max<int64_t>(n, 1) + 8.0;
      continue;
    }
    if (hc.status[STATUS_FACE_OVERFLOW]) {
      if (attempt >= 2) return MV_ERR_CAPACITY;
      face_cap = (int64_t)(hc.face_counter * 1.15) + 4096;
      ctx->face_ratio_hint = (double)face_cap / (double)std::max<int64_t>(n, 1);
      continue;
    }
    F = (int64_t)hc.face_counter;
    stats.cells_built = (int64_t)hc.stats[ST_CELLS];
    stats.neighbours_clipped = (int64_t)hc.stats[ST_NEIGHBOURS];
    stats.planes_added = (int64_t)hc.stats[ST_PLANES];
    stats.f32_undecided = (int64_t)hc.stats[ST_F32_UNDECIDED];
    stats.exact_tests = (int64_t)hc.stats[ST_EXACT];
    stats.extra_shells = (int64_t)hc.stats[ST_SHELLS];
    stats.overflow_cells = (int64_t)hc.stats[ST_OVERFLOW];
    stats.serial_rings = (int64_t)hc.stats[ST_SERIAL_RING];
    break;
  }

  // ---- flatten: faces in cell order (voronoi.rs:226) ----
  {
    size_t FF = (size_t)std::max<int64_t>(F, 1);
    e = 0;
    e |= ensure(ctx, W.f_left, 4 * FF);
    e |= ensure(ctx, W.f_right, 4 * FF);
    e |= ensure(ctx, W.f_area, 8 * FF);
    e |= ensure(ctx, W.f_cen, 24 * FF);
    e |= ensure(ctx, W.f_nrm, 24 * FF);
    e |= ensure(ctx, W.f_code, FF);
    if (e) return MV_ERR_OOM;
  }
  MV_CUDA(cudaEventRecord(ctx->ev[5], st));
  scan_i32_to_i64(P<int32_t>(W.face_count), n, P<int64_t>(W.face_off), P<long long>(W.scan_tmp), st);
  launches += 4;  // scan (3) + reorder
  FaceArrays stage{P<int32_t>(W.st_left), P<int32_t>(W.st_right), P<double>(W.st_area),
                   P<double>(W.st_cen), P<double>(W.st_nrm), P<uint8_t>(W.st_code)};
  FaceArrays fin{P<int32_t>(W.f_left), P<int32_t>(W.f_right), P<double>(W.f_area),
                 P<double>(W.f_cen), P<double>(W.f_nrm), P<uint8_t>(W.f_code)};
  launch_reorder(stage, F, P<int64_t>(W.stage_off), P<int64_t>(W.face_off), fin, st);

  // ---- Voronoi::finalize: cell -> face CSR (voronoi.rs:241-263) ----
  int64_t Cn = 0;
  if (o.face_mode == MV_FACES_OWNED) {
    MV_CUDA(cudaMemsetAsync(W.in_count.p, 0, 4 * N, st));
    MV_CUDA(cudaMemsetAsync(W.cursor.p, 0, 4 * N, st));
    launch_csr_counts(fin, F, P<int32_t>(W.face_count), ni, P<int32_t>(W.in_count),
                      P<int32_t>(W.conn_count), st);
    scan_i32_to_i64(P<int32_t>(W.conn_count), n, P<int64_t>(W.conn_off), P<long long>(W.scan_tmp), st);
    MV_RB(&Cn, P<int64_t>(W.conn_off) + n, 8);
    if (ensure(ctx, W.conn, 4 * (size_t)std::max<int64_t>(Cn, 1))) return MV_ERR_OOM;
    launch_csr_fill(fin, F, P<int64_t>(W.face_off), P<int64_t>(W.conn_off), P<int32_t>(W.in_count),
                    P<int32_t>(W.cursor), ni, P<int32_t>(W.conn), st);
    launches += 7;  // in-count, conn-count, scan (3), fill, sort
  }
  MV_CUDA(cudaEventRecord(ctx->ev[6], st));
  MV_CUDA(cudaGetLastError());
  MV_CUDA(cudaStreamSynchronize(st));
  if (exporting) {
    Job Jx;
    std::memset(&Jx, 0, sizeof(Jx));
    Jx.gen = P<double>(W.gen);
    Jx.sid = P<int32_t>(W.sid);
    for (int k = 0; k < 6; k++)
      for (int i = 0; i < 3; i++) Jx.bp[k][i] = s.bp[k][i];
    for (int c = 0; c < 27; c++) {
      const int m[3] = {c % 3 - 1, (c / 3) % 3 - 1, c / 9 - 1};
      for (int i = 0; i < 3; i++) Jx.shift[c][i] = -((double)(-m[i]) * s.width[i]);
    }
    Jx.rec = P<double>(W.rec);
    Jx.rec_off = P<int64_t>(W.rec_off);
    int rx = export_cells(ctx, Jx, n, cells_flags, st, &launches, cells_out);
    if (rx) return rx;
  }
  stats.device_bytes = (int64_t)ctx->dev_bytes;
  stats.kernel_launches = launches;
  {
    float t01 = 0.f, t12 = 0.f, t34 = 0.f, t56 = 0.f, t78 = 0.f;
    cudaEventElapsedTime(&t01, ctx->ev[0], ctx->ev[1]);
    cudaEventElapsedTime(&t12, ctx->ev[1], ctx->ev[2]);
    if (ctx->large_ran) cudaEventElapsedTime(&t34, ctx->ev[3], ctx->ev[4]);
    if (ctx->retry_ran) cudaEventElapsedTime(&t78, ctx->ev[7], ctx->ev[8]);
    cudaEventElapsedTime(&t56, ctx->ev[5], ctx->ev[6]);
    stats.ms_grid = t01;
    stats.ms_cells = t12 + t34 + t78;
    stats.ms_retry = t78;
    stats.ms_finalize = t56;
  }
  ctx->last = stats;

  out->n_cells = n;
  out->n_faces = F;
  out->n_connections = Cn;
  out->cell_volume = P<double>(W.volume);
  out->cell_centroid = P<double>(W.centroid);
  out->cell_safety_radius = P<double>(W.sr);
  out->cell_face_offset = o.face_mode == MV_FACES_OWNED ? P<int64_t>(W.conn_off) : nullptr;
  out->cell_face_count = o.face_mode == MV_FACES_OWNED ? P<int32_t>(W.conn_count) : nullptr;
  out->face_left = P<int32_t>(W.f_left);
  out->face_right = P<int32_t>(W.f_right);
  out->face_area = P<double>(W.f_area);
  out->face_centroid = P<double>(W.f_cen);
  out->face_normal = P<double>(W.f_nrm);
  out->face_shift_code = P<uint8_t>(W.f_code);
  out->cell_face_connections = o.face_mode == MV_FACES_OWNED ? P<int32_t>(W.conn) : nullptr;
  out->error_cell = -1;
  return MV_OK;
}

// ---- batches (mv_context_build_batch[_device]) ----
// Builds many tessellations at once: per-tessellation setups on the host, one batch
// grid (every tessellation's grid plus an empty end cell, one radix sort), the cell
// phase over all cells with the job table, one finalize whose faces and CSR are then
// made local to each tessellation.
int build_batch_device_impl(mv_context* ctx, const double* d_xyz, const uint8_t* d_mask,
                            const mv_job* jobs, int64_t njobs, const mv_options* opts_in,
                            mv_batch_voronoi* out) {
  mv_options o;
  mv_options_default(&o);
  if (opts_in) o = *opts_in;
  if (!ctx || !out || !jobs || njobs <= 0 || njobs > (1 << 24)) return MV_ERR_ARG;
  std::memset(out, 0, sizeof(*out));
  out->error_job = -1;
  out->error_cell = -1;
  if (o.precision != MV_PRECISION_FP64 && o.precision != MV_PRECISION_FILTERED) return MV_ERR_ARG;
  if (o.face_mode != MV_FACES_OWNED && o.face_mode != MV_FACES_ALL) return MV_ERR_ARG;
  if (o.pipeline < MV_PIPELINE_AUTO || o.pipeline > MV_PIPELINE_FUSED || o.chunk_cells < 0)
    return MV_ERR_ARG;
  const int nj = (int)njobs;
  std::vector<Setup> S(nj);
  std::vector<int32_t> pos(nj + 1), cb(nj + 1);
  std::vector<BatchGrid> bg(nj);
  int64_t ntot = 0, ctot = 0;
  bool any_mask = false;
  double ratio = 0.0;
  for (int j = 0; j < nj; j++) {
    const mv_job& jb = jobs[j];
    if (jb.n < 0 || jb.n >= (int64_t)(0xffffffffu / 27u)) return MV_ERR_ARG;
    int rc = make_setup(jb.n, jb.anchor, jb.width, jb.dimensionality, jb.periodic, o, &S[j]);
    if (rc) return rc;
    pos[j] = (int32_t)ntot;
    cb[j] = (int32_t)ctot;
    ntot += jb.n;
    ctot += (int64_t)S[j].G[0] * S[j].G[1] * S[j].G[2] + 1;
    if (ntot >= INT32_MAX || ctot >= INT32_MAX) return MV_ERR_ARG;
    BatchGrid& g = bg[j];
    std::memset(&g, 0, sizeof(g));
    for (int i = 0; i < 3; i++) g.G[i] = S[j].G[i], g.a[i] = S[j].anchor[i], g.inv[i] = S[j].ginv[i];
    g.dim = S[j].dim;
    g.cbase = cb[j];
    any_mask |= jb.has_mask != 0;
    ratio = std::max(ratio, face_ratio(S[j].dim, o.face_mode));
  }
  pos[nj] = (int32_t)ntot;
  cb[nj] = (int32_t)ctot;
  if ((ntot > 0 && !d_xyz) || (any_mask && !d_mask)) return MV_ERR_ARG;
  MV_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t st = o.stream ? (cudaStream_t)o.stream : ctx->stream;
  Workspace& W = ctx->ws;
  const int ni = (int)ntot;
  const size_t N = (size_t)std::max<int64_t>(ntot, 1);
  const int64_t ncell = ctot;

  // ---- workspace ----
  int e = 0;
  e |= ensure(ctx, W.gen, 24 * N);
  e |= ensure(ctx, W.sx, 8 * N);
  e |= ensure(ctx, W.sy, 8 * N);
  e |= ensure(ctx, W.sz, 8 * N);
  e |= ensure(ctx, W.sid, 4 * N);
  e |= ensure(ctx, W.cid, 4 * N);
  e |= ensure(ctx, W.cell_count, 4 * (ncell + 1));
  e |= ensure(ctx, W.cell_start, 4 * (ncell + 1));
  e |= ensure(ctx, W.dflag, 4 * (ncell + 1));
  e |= ensure(ctx, W.dprefix, 4 * (ncell + 1));
  e |= ensure(ctx, W.scan_tmp, 8 * (scan_tmp_elems(std::max<int64_t>(ncell + 1, N)) + 64));
  e |= ensure(ctx, W.volume, 8 * N);
  e |= ensure(ctx, W.centroid, 24 * N);
  e |= ensure(ctx, W.sr, 8 * N);
  e |= ensure(ctx, W.face_count, 4 * N);
  e |= ensure(ctx, W.stage_off, 8 * N);
  e |= ensure(ctx, W.face_off, 8 * (N + 1));
  e |= ensure(ctx, W.in_count, 4 * N);
  e |= ensure(ctx, W.conn_count, 4 * N);
  e |= ensure(ctx, W.conn_off, 8 * (N + 1));
  e |= ensure(ctx, W.cursor, 4 * N);
  e |= ensure(ctx, W.ovf_a, 4 * N);
  e |= ensure(ctx, W.ovf_b, 4 * N);
  e |= ensure(ctx, W.counters, sizeof(DevCounters));
  e |= ensure(ctx, W.dkey_a, 8 * N);
  e |= ensure(ctx, W.dkey_b, 8 * N);
  e |= ensure(ctx, W.dval_a, 4 * N);
  e |= ensure(ctx, W.dval_b, 4 * N);
  e |= ensure(ctx, W.fkey, 4 * N);
  const size_t sort_bytes = grid_dense_sort_bytes(ni, ncell);
  e |= ensure(ctx, W.dsort_tmp, sort_bytes + 256);
  e |= ensure(ctx, W.b_jobs, sizeof(Job) * (size_t)nj);
  e |= ensure(ctx, W.b_pos, 4 * (size_t)(nj + 1));
  e |= ensure(ctx, W.b_cbase, 4 * (size_t)(nj + 1));
  e |= ensure(ctx, W.b_grid, sizeof(BatchGrid) * (size_t)nj);
  e |= ensure(ctx, W.b_ext_keys, 8 * 6 * (size_t)nj);
  e |= ensure(ctx, W.b_ext, 8 * 6 * (size_t)nj);
  e |= ensure(ctx, W.b_fbase, 8 * (size_t)(nj + 1));
  e |= ensure(ctx, W.b_cbconn, 8 * (size_t)(nj + 1));
  if (e) return MV_ERR_OOM;
  const int32_t* d_pos = P<int32_t>(W.b_pos);
  MV_CUDA(cudaMemcpyAsync(W.b_pos.p, pos.data(), 4 * (size_t)(nj + 1), cudaMemcpyHostToDevice, st));
  MV_CUDA(cudaMemcpyAsync(W.b_cbase.p, cb.data(), 4 * (size_t)(nj + 1), cudaMemcpyHostToDevice, st));
  MV_CUDA(cudaMemcpyAsync(W.b_grid.p, bg.data(), sizeof(BatchGrid) * (size_t)nj, cudaMemcpyHostToDevice, st));
  const int pi = o.precision == MV_PRECISION_FILTERED ? 1 : 0;
  if (ensure(ctx, W.big, big_slot_bytes(ctx, pi, ntot))) return MV_ERR_OOM;
  ratio = std::max(ratio, ctx->face_ratio_hint);
  int64_t face_cap = (int64_t)(ratio * (double)ntot) + 4096;

  DevCounters* C = P<DevCounters>(W.counters);
  mv_build_stats stats{};
  int64_t launches = 0;
  int64_t F = 0;
  std::vector<Job> JJ(nj);
  for (int attempt = 0;; attempt++) {
    size_t FC = (size_t)face_cap;
    e = 0;
    e |= ensure(ctx, W.st_left, 4 * FC);
    e |= ensure(ctx, W.st_right, 4 * FC);
    e |= ensure(ctx, W.st_area, 8 * FC);
    e |= ensure(ctx, W.st_cen, 24 * FC);
    e |= ensure(ctx, W.st_nrm, 24 * FC);
    e |= ensure(ctx, W.st_code, FC);
    if (e) return MV_ERR_OOM;
    face_cap = (int64_t)std::min(W.st_left.cap / 4, W.st_code.cap);
    face_cap = std::min<int64_t>(face_cap, (int64_t)(W.st_area.cap / 8));
    face_cap = std::min<int64_t>(face_cap, (int64_t)(W.st_cen.cap / 24));
    MV_CUDA(cudaMemsetAsync(C, 0, sizeof(DevCounters), st));
    // the failing cell is a minimum over the failing cells: start above every index
    MV_CUDA(cudaMemsetAsync(C->status + STATUS_CELL, 0x7f, sizeof(int32_t), st));
    MV_CUDA(cudaMemsetAsync(W.cell_count.p, 0, 4 * (ncell + 1), st));

    // ---- generators + batch grid ----
    MV_CUDA(cudaEventRecord(ctx->ev[0], st));
    launch_batch_grid(d_xyz, ni, d_pos, P<int32_t>(W.b_cbase), nj, P<BatchGrid>(W.b_grid), ncell,
                      P<double>(W.gen), P<unsigned long long>(W.b_ext_keys), P<double>(W.b_ext),
                      &C->bad_input, P<int32_t>(W.cid), P<int32_t>(W.cell_count),
                      P<int32_t>(W.cell_start), P<int32_t>(W.dflag), P<int32_t>(W.dprefix),
                      P<long long>(W.scan_tmp), st);
    MV_CUDA(launch_batch_sort(P<double>(W.gen), ni, d_pos, P<int32_t>(W.b_cbase), nj, P<BatchGrid>(W.b_grid),
                              ncell, P<int32_t>(W.cid), P<int32_t>(W.dflag), P<unsigned long long>(W.dkey_a),
                              P<unsigned long long>(W.dkey_b), P<int32_t>(W.dval_a), P<int32_t>(W.dval_b),
                              W.dsort_tmp.p, W.dsort_tmp.cap, P<double>(W.sx), P<double>(W.sy),
                              P<double>(W.sz), P<int32_t>(W.sid), P<uint32_t>(W.fkey),
                              P<int32_t>(W.cell_start), st));
    // ext init / prep / finish, cell index, 2 x 3 scan kernels, dense flags, keys, sort,
    // gather, starts
    launches += 19;

    // ---- one Job per tessellation, addressing its slices ----
    for (int j = 0; j < nj; j++) {
      const Setup& sj = S[j];
      Job& J = JJ[j];
      std::memset(&J, 0, sizeof(J));
      const int64_t pb = pos[j], cbj = cb[j];
      J.gen = P<double>(W.gen) + 3 * pb;
      J.sx = P<double>(W.sx) + pb;
      J.sy = P<double>(W.sy) + pb;
      J.sz = P<double>(W.sz) + pb;
      J.sid = P<int32_t>(W.sid) + pb;
      J.cell_start = P<int32_t>(W.cell_start) + cbj;
      J.dprefix = P<int32_t>(W.dprefix) + cbj;
      J.cell_dense = P<int32_t>(W.dflag) + cbj;
      J.fkey = P<uint32_t>(W.fkey) + pb;
      J.mask = jobs[j].has_mask ? d_mask + pb : nullptr;
      J.n = (int32_t)jobs[j].n;
      J.face_mode = o.face_mode;
      J.precision = o.precision;
      set_job_geometry(J, sj);
      J.ext = P<double>(W.b_ext) + 6 * j;
      J.ppc_mean = (double)std::max<int64_t>(jobs[j].n, 1) / (double)(cb[j + 1] - cb[j] - 1);
      J.volume = P<double>(W.volume) + pb;
      J.centroid = P<double>(W.centroid) + 3 * pb;
      J.safety_radius = P<double>(W.sr) + pb;
      J.face_count = P<int32_t>(W.face_count) + pb;
      J.stage_off = P<int64_t>(W.stage_off) + pb;
      J.f_left = P<int32_t>(W.st_left);
      J.f_right = P<int32_t>(W.st_right);
      J.f_area = P<double>(W.st_area);
      J.f_centroid = P<double>(W.st_cen);
      J.f_normal = P<double>(W.st_nrm);
      J.f_code = P<uint8_t>(W.st_code);
      J.face_counter = &C->face_counter;
      J.face_cap = face_cap;
      J.work_counter = &C->work[0];
      J.ovf_list = P<int32_t>(W.ovf_a);
      J.ovf_count = &C->ovf_count[0];
      J.status = C->status;
      J.stats = C->stats;
      J.big = static_cast<char*>(W.big.p);
      J.id_base = (int32_t)pb;
    }
    MV_CUDA(cudaMemcpyAsync(W.b_jobs.p, JJ.data(), sizeof(Job) * (size_t)nj, cudaMemcpyHostToDevice, st));
    // the template Job: shared fields (counters, staging, queues) and the batch's size
    Job J0 = JJ[0];
    J0.n = ni;
    J0.order = nullptr;
    J0.n_order = ni;
    const JobTable TB{P<Job>(W.b_jobs), d_pos, nj};
    DevCounters hc;
    {
      const int rcp = run_cell_phase(ctx, J0, TB, 3, o, ntot, pi, true, false, st, &launches, &stats, &hc);
      if (rcp) return rcp;
    }
    if (hc.status[STATUS_CODE]) {
      const int64_t g = hc.status[STATUS_CELL];
      const int jf = (int)(std::upper_bound(pos.begin(), pos.end() - 1, (int32_t)g) - pos.begin()) - 1;
      out->n_jobs = nj;
      out->error_job = jf;
      out->error_cell = g - pos[std::max(jf, 0)];
      return hc.status[STATUS_CODE];
    }
    if (hc.ovf_count[1] > 0) return MV_ERR_CAPACITY;
    if (hc.status[STATUS_REC_OVERFLOW]) {
      if (attempt >= 2) return MV_ERR_CAPACITY;
      ctx->rec_words_hint = 1.2 * (double)hc.rec_counter / (double)std::max<int64_t>(ntot, 1) + 8.0;
      continue;
    }
    if (hc.status[STATUS_FACE_OVERFLOW]) {
      if (attempt >= 2) return MV_ERR_CAPACITY;
      face_cap = (int64_t)(hc.face_counter * 1.15) + 4096;
      ctx->face_ratio_hint = (double)face_cap / (double)std::max<int64_t>(ntot, 1);
      continue;
    }
    F = (int64_t)hc.face_counter;
    stats.cells_built = (int64_t)hc.stats[ST_CELLS];
    stats.neighbours_clipped = (int64_t)hc.stats[ST_NEIGHBOURS];
    stats.planes_added = (int64_t)hc.stats[ST_PLANES];
    stats.f32_undecided = (int64_t)hc.stats[ST_F32_UNDECIDED];
    stats.exact_tests = (int64_t)hc.stats[ST_EXACT];
    stats.extra_shells = (int64_t)hc.stats[ST_SHELLS];
    stats.overflow_cells = (int64_t)hc.stats[ST_OVERFLOW];
    stats.serial_rings = (int64_t)hc.stats[ST_SERIAL_RING];
    break;
  }

  // ---- flatten + finalize over the batch, then local indices ----
  {
    size_t FF = (size_t)std::max<int64_t>(F, 1);
    e = 0;
    e |= ensure(ctx, W.f_left, 4 * FF);
    e |= ensure(ctx, W.f_right, 4 * FF);
    e |= ensure(ctx, W.f_area, 8 * FF);
    e |= ensure(ctx, W.f_cen, 24 * FF);
    e |= ensure(ctx, W.f_nrm, 24 * FF);
    e |= ensure(ctx, W.f_code, FF);
    if (e) return MV_ERR_OOM;
  }
  MV_CUDA(cudaEventRecord(ctx->ev[5], st));
  scan_i32_to_i64(P<int32_t>(W.face_count), ntot, P<int64_t>(W.face_off), P<long long>(W.scan_tmp), st);
  FaceArrays stage{P<int32_t>(W.st_left), P<int32_t>(W.st_right), P<double>(W.st_area),
                   P<double>(W.st_cen), P<double>(W.st_nrm), P<uint8_t>(W.st_code)};
  FaceArrays fin{P<int32_t>(W.f_left), P<int32_t>(W.f_right), P<double>(W.f_area),
                 P<double>(W.f_cen), P<double>(W.f_nrm), P<uint8_t>(W.f_code)};
  launch_reorder(stage, F, P<int64_t>(W.stage_off), P<int64_t>(W.face_off), fin, st);
  launches += 4;
  int64_t Cn = 0;
  const bool owned = o.face_mode == MV_FACES_OWNED;
  if (owned) {
    MV_CUDA(cudaMemsetAsync(W.in_count.p, 0, 4 * N, st));
    MV_CUDA(cudaMemsetAsync(W.cursor.p, 0, 4 * N, st));
    launch_batch_csr(fin, F, P<int64_t>(W.face_off), P<int32_t>(W.face_count), ni, d_pos, nj,
                     P<int32_t>(W.in_count), P<int32_t>(W.conn_count), st);
    scan_i32_to_i64(P<int32_t>(W.conn_count), ntot, P<int64_t>(W.conn_off), P<long long>(W.scan_tmp), st);
    MV_RB(&Cn, P<int64_t>(W.conn_off) + ntot, 8);
    if (ensure(ctx, W.conn, 4 * (size_t)std::max<int64_t>(Cn, 1))) return MV_ERR_OOM;
    launch_batch_csr_fill(fin, F, P<int64_t>(W.face_off), P<int64_t>(W.conn_off), P<int32_t>(W.in_count),
                          P<int32_t>(W.cursor), ni, d_pos, nj, P<int32_t>(W.conn), st);
    launches += 7;
  }
  launch_batch_localize(fin, F, P<int64_t>(W.face_off), owned ? P<int64_t>(W.conn_off) : nullptr,
                        P<int32_t>(W.conn_count), P<int32_t>(W.conn), ni, d_pos, nj, P<int64_t>(W.b_fbase),
                        P<int64_t>(W.b_cbconn), st);
  launches += owned ? 3 : 2;
  MV_CUDA(cudaEventRecord(ctx->ev[6], st));
  ctx->bj_cell.assign(pos.begin(), pos.end());
  ctx->bj_face.assign(nj + 1, 0);
  ctx->bj_conn.assign(nj + 1, 0);
  MV_RB(ctx->bj_face.data(), W.b_fbase.p, 8 * (size_t)(nj + 1));
  if (owned) MV_RB(ctx->bj_conn.data(), W.b_cbconn.p, 8 * (size_t)(nj + 1));
  MV_CUDA(cudaGetLastError());
  MV_CUDA(cudaStreamSynchronize(st));
  stats.device_bytes = (int64_t)ctx->dev_bytes;
  stats.kernel_launches = launches;
  {
    float t01 = 0.f, t12 = 0.f, t34 = 0.f, t56 = 0.f, t78 = 0.f;
    cudaEventElapsedTime(&t01, ctx->ev[0], ctx->ev[1]);
    cudaEventElapsedTime(&t12, ctx->ev[1], ctx->ev[2]);
    if (ctx->large_ran) cudaEventElapsedTime(&t34, ctx->ev[3], ctx->ev[4]);
    if (ctx->retry_ran) cudaEventElapsedTime(&t78, ctx->ev[7], ctx->ev[8]);
    cudaEventElapsedTime(&t56, ctx->ev[5], ctx->ev[6]);
    stats.ms_grid = t01;
    stats.ms_cells = t12 + t34 + t78;
    stats.ms_retry = t78;
    stats.ms_finalize = t56;
  }
  ctx->last = stats;
  out->n_jobs = nj;
  out->n_cells = ntot;
  out->n_faces = F;
  out->n_connections = Cn;
  out->job_cell_offset = ctx->bj_cell.data();
  out->job_face_offset = ctx->bj_face.data();
  out->job_connection_offset = ctx->bj_conn.data();
  out->cell_volume = P<double>(W.volume);
  out->cell_centroid = P<double>(W.centroid);
  out->cell_safety_radius = P<double>(W.sr);
  out->cell_face_offset = owned ? P<int64_t>(W.conn_off) : nullptr;
  out->cell_face_count = owned ? P<int32_t>(W.conn_count) : nullptr;
  out->face_left = P<int32_t>(W.f_left);
  out->face_right = P<int32_t>(W.f_right);
  out->face_area = P<double>(W.f_area);
  out->face_centroid = P<double>(W.f_cen);
  out->face_normal = P<double>(W.f_nrm);
  out->face_shift_code = P<uint8_t>(W.f_code);
  out->cell_face_connections = owned ? P<int32_t>(W.conn) : nullptr;
  return MV_OK;
}

struct HostLayout {
  size_t off[16];
  size_t total;
};

HostLayout host_layout(int64_t n, int64_t F, int64_t Cn) {
  const size_t sz[] = {8 * (size_t)n,  24 * (size_t)n, 8 * (size_t)n,  8 * (size_t)n,
                       4 * (size_t)n,  4 * (size_t)F,  4 * (size_t)F,  8 * (size_t)F,
                       24 * (size_t)F, 24 * (size_t)F, (size_t)F,      4 * (size_t)Cn};
  HostLayout L;
  size_t o = 0;
  for (int i = 0; i < 12; i++) {
    L.off[i] = o;
    o += (sz[i] + 255) & ~(size_t)255;
  }
  L.total = o;
  return L;
}

int copy_to_host(mv_context* ctx, const mv_device_voronoi& d, int64_t n, const Setup& s,
                 cudaStream_t st, mv_voronoi* hv) {
  HostLayout L = host_layout(n, d.n_faces, d.n_connections);
  if (ctx->host_cap < L.total) {
    if (ctx->host) cudaFreeHost(ctx->host);
    ctx->host = nullptr;
    ctx->host_cap = 0;
    size_t want = L.total + L.total / 8 + 4096;
    if (cudaHostAlloc(&ctx->host, want, cudaHostAllocDefault) != cudaSuccess) {
      cudaGetLastError();
      ctx->host = nullptr;
      return MV_ERR_OOM;
    }
    ctx->host_cap = want;
  }
  char* b = static_cast<char*>(ctx->host);
  std::memset(hv, 0, sizeof(*hv));
  hv->n_cells = n;
  hv->n_faces = d.n_faces;
  hv->n_connections = d.n_connections;
  hv->dimensionality = s.dim;
  hv->periodic = s.periodic;
  for (int i = 0; i < 3; i++) hv->anchor[i] = s.anchor[i], hv->width[i] = s.width[i];
  hv->cell_volume = (double*)(b + L.off[0]);
  hv->cell_centroid = (double*)(b + L.off[1]);
  hv->cell_safety_radius = (double*)(b + L.off[2]);
  hv->cell_face_offset = (int64_t*)(b + L.off[3]);
  hv->cell_face_count = (int32_t*)(b + L.off[4]);
  hv->face_left = (int32_t*)(b + L.off[5]);
  hv->face_right = (int32_t*)(b + L.off[6]);
  hv->face_area = (double*)(b + L.off[7]);
  hv->face_centroid = (double*)(b + L.off[8]);
  hv->face_normal = (double*)(b + L.off[9]);
  hv->face_shift_code = (uint8_t*)(b + L.off[10]);
  hv->cell_face_connections = (int32_t*)(b + L.off[11]);
  hv->error_cell = -1;
  auto cp = [&](void* dst, const void* src, size_t bytes) -> cudaError_t {
    if (!bytes || !src) return cudaSuccess;
    return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st);
  };
  const size_t N = (size_t)n, F = (size_t)d.n_faces, Cn = (size_t)d.n_connections;
  MV_CUDA(cp(hv->cell_volume, d.cell_volume, 8 * N));
  MV_CUDA(cp(hv->cell_centroid, d.cell_centroid, 24 * N));
  MV_CUDA(cp(hv->cell_safety_radius, d.cell_safety_radius, 8 * N));
  MV_CUDA(cp(hv->cell_face_offset, d.cell_face_offset, 8 * N));
  MV_CUDA(cp(hv->cell_face_count, d.cell_face_count, 4 * N));
  MV_CUDA(cp(hv->face_left, d.face_left, 4 * F));
  MV_CUDA(cp(hv->face_right, d.face_right, 4 * F));
  MV_CUDA(cp(hv->face_area, d.face_area, 8 * F));
  MV_CUDA(cp(hv->face_centroid, d.face_centroid, 24 * F));
  MV_CUDA(cp(hv->face_normal, d.face_normal, 24 * F));
  MV_CUDA(cp(hv->face_shift_code, d.face_shift_code, F));
  MV_CUDA(cp(hv->cell_face_connections, d.cell_face_connections, 4 * Cn));
  MV_CUDA(cudaStreamSynchronize(st));
  if (!d.cell_face_offset) {
    hv->cell_face_offset = nullptr;
    hv->cell_face_count = nullptr;
    hv->cell_face_connections = nullptr;
  }
  return MV_OK;
}

// The cells of a cells build into the context's second pinned arena.
int copy_cells_to_host(mv_context* ctx, const mv_cells& d, cudaStream_t st, mv_cells* h) {
  const int64_t n = d.n_cells, P_ = d.n_planes, V = d.n_vertices, T = d.n_tets, Fc = d.n_faces,
                FV = d.n_face_vertices;
  const bool tets = d.tet_vertices != nullptr, faces = d.face_vertices != nullptr;
  const size_t sz[] = {8 * (size_t)(n + 1), 24 * (size_t)P_, 24 * (size_t)P_, 4 * (size_t)P_,
                       (size_t)P_, 8 * (size_t)(n + 1), 24 * (size_t)V, 12 * (size_t)V,
                       tets ? 8 * (size_t)(n + 1) : 0, 72 * (size_t)T, 4 * (size_t)T,
                       faces ? 8 * (size_t)(n + 1) : 0, 4 * (size_t)Fc,
                       faces ? 8 * (size_t)(Fc + 1) : 0, 4 * (size_t)FV};
  const int K = (int)(sizeof(sz) / sizeof(sz[0]));
  size_t offs[16], total = 0;
  for (int i = 0; i < K; i++) {
    offs[i] = total;
    total += (sz[i] + 255) & ~(size_t)255;
  }
  if (ctx->host_cells_cap < total) {
    if (ctx->host_cells) cudaFreeHost(ctx->host_cells);
    ctx->host_cells = nullptr;
    ctx->host_cells_cap = 0;
    const size_t want = total + total / 8 + 4096;
    if (cudaHostAlloc(&ctx->host_cells, want, cudaHostAllocDefault) != cudaSuccess) {
      cudaGetLastError();
      ctx->host_cells = nullptr;
      return MV_ERR_OOM;
    }
    ctx->host_cells_cap = want;
  }
  char* b = static_cast<char*>(ctx->host_cells);
  const void* src[] = {d.cell_plane_offset, d.plane_normal, d.plane_point, d.plane_right,
                       d.plane_shift_code, d.cell_vertex_offset, d.vertex_loc, d.vertex_dual,
                       d.cell_tet_offset, d.tet_vertices, d.tet_plane, d.cell_face_offset,
                       d.face_plane, d.face_vertex_offset, d.face_vertices};
  for (int i = 0; i < K; i++)
    if (sz[i] && src[i]) MV_CUDA(cudaMemcpyAsync(b + offs[i], src[i], sz[i], cudaMemcpyDeviceToHost, st));
  MV_CUDA(cudaStreamSynchronize(st));
  *h = d;
  auto at = [&](int i, const void* p) -> char* { return p ? b + offs[i] : nullptr; };
  h->cell_plane_offset = (int64_t*)at(0, d.cell_plane_offset);
  h->plane_normal = (double*)at(1, d.plane_normal);
  h->plane_point = (double*)at(2, d.plane_point);
  h->plane_right = (int32_t*)at(3, d.plane_right);
  h->plane_shift_code = (uint8_t*)at(4, d.plane_shift_code);
  h->cell_vertex_offset = (int64_t*)at(5, d.cell_vertex_offset);
  h->vertex_loc = (double*)at(6, d.vertex_loc);
  h->vertex_dual = (int32_t*)at(7, d.vertex_dual);
  h->cell_tet_offset = (int64_t*)at(8, d.cell_tet_offset);
  h->tet_vertices = (double*)at(9, d.tet_vertices);
  h->tet_plane = (int32_t*)at(10, d.tet_plane);
  h->cell_face_offset = (int64_t*)at(11, d.cell_face_offset);
  h->face_plane = (int32_t*)at(12, d.face_plane);
  h->face_vertex_offset = (int64_t*)at(13, d.face_vertex_offset);
  h->face_vertices = (int32_t*)at(14, d.face_vertices);
  return MV_OK;
}

// Builds with host buffers run their GPU phase (input copy, kernels) one at a time per
// device and copy their results back outside it: with several contexts on one device
// (one per host thread), one build's result copy then overlaps the next build's
// kernels, instead of all builds computing side by side and copying at once.
constexpr int MAX_PHASE_DEVICES = 64;
std::mutex g_gpu_phase[MAX_PHASE_DEVICES];

struct GpuPhase {
  std::mutex* m;
  explicit GpuPhase(int device)
      : m(device >= 0 && device < MAX_PHASE_DEVICES ? &g_gpu_phase[device] : nullptr) {
    if (m) m->lock();
  }
  void release() {
    if (m) m->unlock();
    m = nullptr;
  }
  ~GpuPhase() { release(); }
};

int build_host_impl(mv_context* ctx, const double* xyz, const uint8_t* mask, int64_t n,
                    const double* anchor, const double* width, int dim, int periodic,
                    const mv_options* opts, mv_voronoi** out, int cells_flags = -1,
                    mv_cells** cells_out = nullptr) {
  if (!ctx || !out || n < 0 || (n > 0 && !xyz)) return MV_ERR_ARG;
  mv_options o;
  mv_options_default(&o);
  if (opts) o = *opts;
  Setup s;
  int rc = make_setup(n, anchor, width, dim, periodic, o, &s);
  if (rc) return rc;
  MV_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t st = o.stream ? (cudaStream_t)o.stream : ctx->stream;
  GpuPhase phase(ctx->device);
  const size_t N = (size_t)std::max<int64_t>(n, 1);
  if (ensure(ctx, ctx->ws.in_xyz, 24 * N) || ensure(ctx, ctx->ws.in_mask, N)) return MV_ERR_OOM;
  if (n > 0) MV_CUDA(cudaMemcpyAsync(ctx->ws.in_xyz.p, xyz, 24 * (size_t)n, cudaMemcpyHostToDevice, st));
  if (mask && n > 0) MV_CUDA(cudaMemcpyAsync(ctx->ws.in_mask.p, mask, (size_t)n, cudaMemcpyHostToDevice, st));
  mv_device_voronoi d{};
  d.error_cell = -1;
  mv_cells dc{};
  rc = build_device_impl(ctx, P<double>(ctx->ws.in_xyz), mask ? P<uint8_t>(ctx->ws.in_mask) : nullptr,
                         n, anchor, width, dim, periodic, &o, &d, cells_flags,
                         cells_flags >= 0 ? &dc : nullptr);
  if (rc) {
    std::memset(&ctx->hv, 0, sizeof(ctx->hv));
    ctx->hv.n_cells = n;
    ctx->hv.error_cell = d.error_cell;
    *out = &ctx->hv;
    return rc;
  }
  phase.release();
  rc = copy_to_host(ctx, d, n, s, st, &ctx->hv);
  if (rc) return rc;
  *out = &ctx->hv;
  if (cells_flags >= 0) {
    rc = copy_cells_to_host(ctx, dc, st, &ctx->hc);
    if (rc) return rc;
    *cells_out = &ctx->hc;
  }
  return MV_OK;
}

// Batch build with host inputs: inputs copied to the device, the result copied into the
// context's pinned host arena (same layout as a single build's).
int build_batch_host_impl(mv_context* ctx, const double* xyz, const uint8_t* mask, const mv_job* jobs,
                          int64_t njobs, const mv_options* opts, mv_batch_voronoi* out) {
  if (!ctx || !out || !jobs || njobs <= 0) return MV_ERR_ARG;
  mv_options o;
  mv_options_default(&o);
  if (opts) o = *opts;
  int64_t ntot = 0;
  bool any_mask = false;
  for (int64_t j = 0; j < njobs; j++) {
    if (jobs[j].n < 0) return MV_ERR_ARG;
    ntot += jobs[j].n;
    any_mask |= jobs[j].has_mask != 0;
  }
  if ((ntot > 0 && !xyz) || (any_mask && !mask)) return MV_ERR_ARG;
  MV_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t st = o.stream ? (cudaStream_t)o.stream : ctx->stream;
  GpuPhase phase(ctx->device);
  const size_t N = (size_t)std::max<int64_t>(ntot, 1);
  if (ensure(ctx, ctx->ws.in_xyz, 24 * N) || ensure(ctx, ctx->ws.in_mask, N)) return MV_ERR_OOM;
  if (ntot > 0)
    MV_CUDA(cudaMemcpyAsync(ctx->ws.in_xyz.p, xyz, 24 * (size_t)ntot, cudaMemcpyHostToDevice, st));
  if (any_mask && ntot > 0)
    MV_CUDA(cudaMemcpyAsync(ctx->ws.in_mask.p, mask, (size_t)ntot, cudaMemcpyHostToDevice, st));
  mv_batch_voronoi d;
  std::memset(&d, 0, sizeof(d));
  d.error_job = -1;
  d.error_cell = -1;
  int rc = build_batch_device_impl(ctx, P<double>(ctx->ws.in_xyz),
                                   any_mask ? P<uint8_t>(ctx->ws.in_mask) : nullptr, jobs, njobs, &o, &d);
  if (rc) {
    *out = d;
    return rc;
  }
  phase.release();
  HostLayout L = host_layout(d.n_cells, d.n_faces, d.n_connections);
  if (ctx->host_cap < L.total) {
    if (ctx->host) cudaFreeHost(ctx->host);
    ctx->host = nullptr;
    ctx->host_cap = 0;
    const size_t want = L.total + L.total / 8 + 4096;
    if (cudaHostAlloc(&ctx->host, want, cudaHostAllocDefault) != cudaSuccess) {
      cudaGetLastError();
      ctx->host = nullptr;
      return MV_ERR_OOM;
    }
    ctx->host_cap = want;
  }
  char* b = static_cast<char*>(ctx->host);
  *out = d;
  out->cell_volume = (double*)(b + L.off[0]);
  out->cell_centroid = (double*)(b + L.off[1]);
  out->cell_safety_radius = (double*)(b + L.off[2]);
  out->cell_face_offset = d.cell_face_offset ? (int64_t*)(b + L.off[3]) : nullptr;
  out->cell_face_count = d.cell_face_count ? (int32_t*)(b + L.off[4]) : nullptr;
  out->face_left = (int32_t*)(b + L.off[5]);
  out->face_right = (int32_t*)(b + L.off[6]);
  out->face_area = (double*)(b + L.off[7]);
  out->face_centroid = (double*)(b + L.off[8]);
  out->face_normal = (double*)(b + L.off[9]);
  out->face_shift_code = (uint8_t*)(b + L.off[10]);
  out->cell_face_connections = d.cell_face_connections ? (int32_t*)(b + L.off[11]) : nullptr;
  auto cp = [&](void* dst, const void* src, size_t bytes) -> cudaError_t {
    if (!bytes || !src || !dst) return cudaSuccess;
    return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st);
  };
  const size_t n = (size_t)d.n_cells, F = (size_t)d.n_faces, Cn = (size_t)d.n_connections;
  MV_CUDA(cp(out->cell_volume, d.cell_volume, 8 * n));
  MV_CUDA(cp(out->cell_centroid, d.cell_centroid, 24 * n));
  MV_CUDA(cp(out->cell_safety_radius, d.cell_safety_radius, 8 * n));
  MV_CUDA(cp(out->cell_face_offset, d.cell_face_offset, 8 * n));
  MV_CUDA(cp(out->cell_face_count, d.cell_face_count, 4 * n));
  MV_CUDA(cp(out->face_left, d.face_left, 4 * F));
  MV_CUDA(cp(out->face_right, d.face_right, 4 * F));
  MV_CUDA(cp(out->face_area, d.face_area, 8 * F));
  MV_CUDA(cp(out->face_centroid, d.face_centroid, 24 * F));
  MV_CUDA(cp(out->face_normal, d.face_normal, 24 * F));
  MV_CUDA(cp(out->face_shift_code, d.face_shift_code, F));
  MV_CUDA(cp(out->cell_face_connections, d.cell_face_connections, 4 * Cn));
  MV_CUDA(cudaStreamSynchronize(st));
  return MV_OK;
}

struct OwnedVoronoi {
  mv_voronoi v;
  void* block;
};

int standalone(const double* xyz, const uint8_t* mask, int64_t n, const double* anchor,
               const double* width, int dim, int periodic, const mv_options* opts,
               mv_voronoi** out) {
  if (!out) return MV_ERR_ARG;
  *out = nullptr;
  mv_context* ctx = nullptr;
  int rc = mv_context_create(-1, &ctx);
  if (rc) return rc;
  mv_voronoi* hv = nullptr;
  rc = build_host_impl(ctx, xyz, mask, n, anchor, width, dim, periodic, opts, &hv);
  OwnedVoronoi* ov = new (std::nothrow) OwnedVoronoi();
  if (!ov) {
    mv_context_destroy(ctx);
    return MV_ERR_OOM;
  }
  ov->v = *hv;
  ov->block = nullptr;
  ov->v._owner = ov;
  if (rc == MV_OK) {
    HostLayout L = host_layout(hv->n_cells, hv->n_faces, hv->n_connections);
    ov->block = std::malloc(std::max<size_t>(L.total, 16));
    if (!ov->block) {
      delete ov;
      mv_context_destroy(ctx);
      return MV_ERR_OOM;
    }
    std::memcpy(ov->block, ctx->host, L.total);
    char* b = static_cast<char*>(ov->block);
    auto rebase = [&](void* p) -> char* {
      return p ? b + (static_cast<char*>(p) - static_cast<char*>(ctx->host)) : nullptr;
    };
    ov->v.cell_volume = (double*)rebase(hv->cell_volume);
    ov->v.cell_centroid = (double*)rebase(hv->cell_centroid);
    ov->v.cell_safety_radius = (double*)rebase(hv->cell_safety_radius);
    ov->v.cell_face_offset = (int64_t*)rebase(hv->cell_face_offset);
    ov->v.cell_face_count = (int32_t*)rebase(hv->cell_face_count);
    ov->v.face_left = (int32_t*)rebase(hv->face_left);
    ov->v.face_right = (int32_t*)rebase(hv->face_right);
    ov->v.face_area = (double*)rebase(hv->face_area);
    ov->v.face_centroid = (double*)rebase(hv->face_centroid);
    ov->v.face_normal = (double*)rebase(hv->face_normal);
    ov->v.face_shift_code = (uint8_t*)rebase(hv->face_shift_code);
    ov->v.cell_face_connections = (int32_t*)rebase(hv->cell_face_connections);
  }
  mv_context_destroy(ctx);
  *out = &ov->v;
  return rc;
}

}  // namespace

extern "C" {

void mv_options_default(mv_options* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->precision = MV_PRECISION_FILTERED;
  o->face_mode = MV_FACES_OWNED;
}

const char* mv_strerror(int s) {
  switch (s) {
    case MV_OK: return "ok";
    case MV_ERR_ARG: return "invalid argument";
    case MV_ERR_DEGENERATE: return "Degenerate point set! (duplicate generators)";
    case MV_ERR_RING: return "No suitable vertex found to extend boundary!";
    case MV_ERR_DET: return "Degenerate 3-plane intersection!";
    case MV_ERR_CAPACITY: return "a cell exceeded the largest device capacity tier";
    case MV_ERR_CUDA: return "CUDA runtime error";
    case MV_ERR_NO_DEVICE: return "no usable CUDA device";
    case MV_ERR_OOM: return "out of device or pinned host memory";
    default: return "unknown status";
  }
}

const char* mv_version(void) { return "mvgpu 0.1.0 (sm_100a)"; }

int mv_context_create(int device, mv_context** out) {
  if (!out) return MV_ERR_ARG;
  *out = nullptr;
  int dev = device;
  if (dev < 0) {
    if (cudaGetDevice(&dev) != cudaSuccess) {
      cudaGetLastError();
      return MV_ERR_NO_DEVICE;
    }
  }
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || dev >= count) {
    cudaGetLastError();
    return MV_ERR_NO_DEVICE;
  }
  MV_CUDA(cudaSetDevice(dev));
  mv_context* ctx = new (std::nothrow) mv_context();
  if (!ctx) return MV_ERR_OOM;
  ctx->device = dev;
  cudaError_t e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, dev);
  for (int i = 0; i < 10 && e == cudaSuccess; i++) e = cudaEventCreate(&ctx->ev[i]);
  // the readback buffer; without it readbacks fall back to cudaMemcpy
  if (e == cudaSuccess) {
    if (cudaHostAlloc(&ctx->rb_host, READBACK_BYTES, cudaHostAllocMapped) != cudaSuccess ||
        cudaHostGetDevicePointer(&ctx->rb_dev, ctx->rb_host, 0) != cudaSuccess) {
      cudaGetLastError();
      if (ctx->rb_host) cudaFreeHost(ctx->rb_host);
      ctx->rb_host = nullptr;
      ctx->rb_dev = nullptr;
    }
  }
  if (e != cudaSuccess) {
    delete ctx;
    return cuda_status(e);
  }
  for (int p = 0; p < 2; p++) {
    ctx->bps_fast[p] = cells_blocks_per_sm_fast(p);
    ctx->bps_large[p] = cells_blocks_per_sm_large(p);
    for (int k = 0; k < 4; k++) ctx->bps_stage[k][p] = stage_blocks_per_sm(k, p);
  }
  if (cudaGetLastError() != cudaSuccess || ctx->bps_fast[0] <= 0 || ctx->bps_fast[1] <= 0) {
    cudaStreamDestroy(ctx->stream);
    delete ctx;
    return MV_ERR_CUDA;
  }
  *out = ctx;
  return MV_OK;
}

void mv_context_destroy(mv_context* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  DevBuf* bufs = reinterpret_cast<DevBuf*>(&ctx->ws);
  const size_t nb = sizeof(Workspace) / sizeof(DevBuf);
  for (size_t i = 0; i < nb; i++)
    if (bufs[i].p) cudaFree(bufs[i].p);
  if (ctx->host) cudaFreeHost(ctx->host);
  if (ctx->host_cells) cudaFreeHost(ctx->host_cells);
  if (ctx->rb_host) cudaFreeHost(ctx->rb_host);
  for (cudaEvent_t ev : ctx->stage_ev) cudaEventDestroy(ev);
  for (int i = 0; i < 10; i++)
    if (ctx->ev[i]) cudaEventDestroy(ctx->ev[i]);
  cudaStreamDestroy(ctx->stream);
  delete ctx;
}

int mv_context_last_stats(const mv_context* ctx, mv_build_stats* out) {
  if (!ctx || !out) return MV_ERR_ARG;
  *out = ctx->last;
  return MV_OK;
}

int mv_context_build_device(mv_context* ctx, const double* d_generators, const uint8_t* d_mask,
                            int64_t n, const double anchor[3], const double width[3],
                            int dimensionality, int periodic, const mv_options* opts,
                            mv_device_voronoi* out) {
  if (!ctx || !anchor || !width) return MV_ERR_ARG;
  return build_device_impl(ctx, d_generators, d_mask, n, anchor, width, dimensionality, periodic,
                           opts, out);
}

int mv_context_build(mv_context* ctx, const double* generators, const uint8_t* mask, int64_t n,
                     const double anchor[3], const double width[3], int dimensionality,
                     int periodic, const mv_options* opts, mv_voronoi** out) {
  if (!anchor || !width) return MV_ERR_ARG;
  return build_host_impl(ctx, generators, mask, n, anchor, width, dimensionality, periodic, opts,
                         out);
}

int mv_context_build_cells_device(mv_context* ctx, const double* d_generators,
                                  const uint8_t* d_mask, int64_t n, const double anchor[3],
                                  const double width[3], int dimensionality, int periodic,
                                  const mv_options* opts, int cells_flags,
                                  mv_device_voronoi* voronoi, mv_cells* cells) {
  if (!ctx || !anchor || !width || !cells || cells_flags < 0) return MV_ERR_ARG;
  return build_device_impl(ctx, d_generators, d_mask, n, anchor, width, dimensionality, periodic,
                           opts, voronoi, cells_flags, cells);
}

int mv_context_build_cells(mv_context* ctx, const double* generators, const uint8_t* mask,
                           int64_t n, const double anchor[3], const double width[3],
                           int dimensionality, int periodic, const mv_options* opts,
                           int cells_flags, mv_voronoi** voronoi, mv_cells** cells) {
  if (!anchor || !width || !cells || cells_flags < 0) return MV_ERR_ARG;
  return build_host_impl(ctx, generators, mask, n, anchor, width, dimensionality, periodic, opts,
                         voronoi, cells_flags, cells);
}

int mv_voronoi_build(const double* generators, int64_t n, const double anchor[3],
                     const double width[3], int dimensionality, int periodic,
                     const mv_options* opts, mv_voronoi** out) {
  if (!anchor || !width) return MV_ERR_ARG;
  return standalone(generators, nullptr, n, anchor, width, dimensionality, periodic, opts, out);
}

int mv_voronoi_build_partial(const double* generators, const uint8_t* mask, int64_t n,
                             const double anchor[3], const double width[3], int dimensionality,
                             int periodic, const mv_options* opts, mv_voronoi** out) {
  if (!anchor || !width || (n > 0 && !mask)) return MV_ERR_ARG;
  return standalone(generators, mask, n, anchor, width, dimensionality, periodic, opts, out);
}

int mv_context_build_batch_device(mv_context* ctx, const double* d_generators, const uint8_t* d_mask,
                                  const mv_job* jobs, int64_t n_jobs, const mv_options* opts,
                                  mv_batch_voronoi* out) {
  return build_batch_device_impl(ctx, d_generators, d_mask, jobs, n_jobs, opts, out);
}

int mv_context_build_batch(mv_context* ctx, const double* generators, const uint8_t* mask,
                           const mv_job* jobs, int64_t n_jobs, const mv_options* opts,
                           mv_batch_voronoi* out) {
  return build_batch_host_impl(ctx, generators, mask, jobs, n_jobs, opts, out);
}

void mv_voronoi_free(mv_voronoi* v) {
  if (!v || !v->_owner) return;
  OwnedVoronoi* ov = static_cast<OwnedVoronoi*>(v->_owner);
  std::free(ov->block);
  delete ov;
}

void mv_shift_from_code(int code, const double width[3], double out[3]) {
  D3 s = shift_of_code(code, width);
  out[0] = s.x, out[1] = s.y, out[2] = s.z;
}

}  // extern "C"
