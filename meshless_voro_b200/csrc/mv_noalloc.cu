// mv_noalloc.cu -- a Voronoi build that allocates nothing.
//
// Some callers cannot call cudaMalloc: a host framework that has handed all device
// memory to its own pool allocator, code that must never trigger the implicit device
// synchronisation of cudaMalloc / cudaFree, or an embedding with a fixed, pre-budgeted
// memory plan.  mv_voronoi_build_noalloc serves them: the caller passes device inputs
// and device outputs, and every scratch buffer of the build (generator copies, the
// uniform grid, face staging, counters) lives in one file-scope static __device__
// array of fixed size, so the build calls no allocating routine at all.
//
// The array bounds the problem size (MV_NOALLOC_MAX_GENERATORS generators).  Every GPU
// that loads the library holds the array until the process exits.  All calls share the
// array, and it keeps the contents of the last call: each call clears what must start
// at zero, and calls that overlap on the GPU (different streams or host threads) race
// on it.
//
// Compared with a context build, the fused kernel's fast tier runs without staging
// slots for very large neighbour shells (a cell whose shell does not narrow into shared
// memory moves to the large tier), and the large tier runs on NA_BIG_SLOTS warps, each
// with one slot inside the array, so it takes the same shells as a context build's
// large tier.  Results are the same; only such cells take longer.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <mutex>

#include "../../include/mvgpu.h"
#include "mv_cell_common.cuh"
#include "mv_internal.h"

namespace mv {
cudaError_t launch_cells(const Job& J, bool large, int blocks, cudaStream_t st, const JobTable& TB);
int cells_blocks_per_sm_fast(int precision);
int cells_blocks_per_sm_large(int precision);
void launch_prep(const double* xyz, int n, int dim, double* gen, unsigned long long* ext_keys,
                 double* ext, int* bad, cudaStream_t st);
void launch_grid(const double* gen, int n, const int G[3], const double a[3], const double inv[3],
                 int32_t* cid, int32_t* count, int32_t* start, int32_t* fill, double* sx, double* sy,
                 double* sz, int32_t* sid, long long* scan_tmp, cudaStream_t st);
void scan_i32_to_i64(const int32_t* in, int64_t n, int64_t* out, long long* tmp, cudaStream_t st);
void launch_reorder(const FaceArrays& stage, int64_t F, const int64_t* stage_off,
                    const int64_t* face_off, const FaceArrays& out, cudaStream_t st);
void launch_csr_counts(const FaceArrays& f, int64_t F, const int32_t* face_count, int n,
                       int32_t* in_count, int32_t* conn_count, cudaStream_t st);
void launch_csr_fill(const FaceArrays& f, int64_t F, const int64_t* face_off, const int64_t* conn_off,
                     const int32_t* in_count, int32_t* cursor, int n, int32_t* conn, cudaStream_t st);
}  // namespace mv

using namespace mv;

namespace {

constexpr int64_t NMAX = MV_NOALLOC_MAX_GENERATORS;
constexpr int64_t CELLMAX = 2 * NMAX;                    // uniform-grid cells
constexpr int64_t FACEMAX = MV_NOALLOC_FACES_PER_GENERATOR * NMAX;  // staged faces
constexpr int64_t SCANMAX = (std::max(CELLMAX + 1, NMAX + 1) + 4095) / 4096 + 64;
constexpr int NA_BIG_SLOTS = 8;  // large-tier warps, one big-shell staging slot each

constexpr size_t al(size_t b) { return (b + 255) & ~(size_t)255; }

// byte offsets of the scratch regions
constexpr size_t O_GEN = 0;
constexpr size_t O_SX = O_GEN + al(24 * NMAX);
constexpr size_t O_SY = O_SX + al(8 * NMAX);
constexpr size_t O_SZ = O_SY + al(8 * NMAX);
constexpr size_t O_SID = O_SZ + al(8 * NMAX);
constexpr size_t O_CID = O_SID + al(4 * NMAX);
constexpr size_t O_CCOUNT = O_CID + al(4 * NMAX);
constexpr size_t O_CSTART = O_CCOUNT + al(4 * (CELLMAX + 1));
constexpr size_t O_CFILL = O_CSTART + al(4 * (CELLMAX + 1));
constexpr size_t O_SCAN = O_CFILL + al(4 * (CELLMAX + 1));
constexpr size_t O_FCOUNT = O_SCAN + al(8 * SCANMAX);
constexpr size_t O_STOFF = O_FCOUNT + al(4 * NMAX);
constexpr size_t O_FOFF = O_STOFF + al(8 * NMAX);
constexpr size_t O_INCNT = O_FOFF + al(8 * (NMAX + 1));
constexpr size_t O_CURSOR = O_INCNT + al(4 * NMAX);
constexpr size_t O_CONNOFF = O_CURSOR + al(4 * NMAX);
constexpr size_t O_OVFA = O_CONNOFF + al(8 * (NMAX + 1));
constexpr size_t O_OVFB = O_OVFA + al(4 * NMAX);
constexpr size_t O_STLEFT = O_OVFB + al(4 * NMAX);
constexpr size_t O_STRIGHT = O_STLEFT + al(4 * FACEMAX);
constexpr size_t O_STAREA = O_STRIGHT + al(4 * FACEMAX);
constexpr size_t O_STCEN = O_STAREA + al(8 * FACEMAX);
constexpr size_t O_STNRM = O_STCEN + al(24 * FACEMAX);
constexpr size_t O_STCODE = O_STNRM + al(24 * FACEMAX);
constexpr size_t O_BIG = O_STCODE + al(FACEMAX);
constexpr size_t O_COUNTERS = O_BIG + al(NA_BIG_SLOTS * BIG_SLOT_BYTES);
constexpr size_t SCRATCH_BYTES = O_COUNTERS + al(sizeof(DevCounters));

// The scratch of every no-alloc build on this GPU.  Host code must not use this name
// as a device address (it is a host-side shadow); it takes the address from
// cudaGetSymbolAddress once per device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[SCRATCH_BYTES];

constexpr int MAX_DEVICES = 64;
struct DeviceSetup {
  unsigned char* base = nullptr;
  int sm_count = 0;
  int bps_fast[2] = {0, 0};
  int bps_large[2] = {0, 0};
};
DeviceSetup g_setup[MAX_DEVICES];
std::mutex g_setup_mutex;

int cuda_status(cudaError_t e) {
  if (e == cudaSuccess) return MV_OK;
  if (e == cudaErrorMemoryAllocation) return MV_ERR_OOM;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return MV_ERR_NO_DEVICE;
  return MV_ERR_CUDA;
}

#define NA_CUDA(call)                              \
  do {                                             \
    cudaError_t e_ = (call);                       \
    if (e_ != cudaSuccess) return cuda_status(e_); \
  } while (0)

// Once per device, with that device current: the device address of the scratch array
// and the launch shape of the cell kernels.
int device_setup(int dev, DeviceSetup** out) {
  if (dev < 0 || dev >= MAX_DEVICES) return MV_ERR_NO_DEVICE;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  DeviceSetup& s = g_setup[dev];
  if (!s.base) {
    void* ptr = nullptr;
    NA_CUDA(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
    NA_CUDA(cudaDeviceGetAttribute(&s.sm_count, cudaDevAttrMultiProcessorCount, dev));
    for (int p = 0; p < 2; p++) {
      s.bps_fast[p] = cells_blocks_per_sm_fast(p);
      s.bps_large[p] = cells_blocks_per_sm_large(p);
    }
    NA_CUDA(cudaGetLastError());
    if (s.bps_fast[0] <= 0 || s.bps_fast[1] <= 0) return MV_ERR_CUDA;
    s.base = static_cast<unsigned char*>(ptr);
  }
  *out = &s;
  return MV_OK;
}

template <class T>
T* at(unsigned char* base, size_t off) {
  return reinterpret_cast<T*>(base + off);
}

}  // namespace

extern "C" int mv_voronoi_build_noalloc(const double* d_generators, const uint8_t* d_mask,
                                        int64_t n, const double anchor[3], const double width[3],
                                        int dimensionality, int periodic, const mv_options* opts_in,
                                        mv_device_voronoi* out, int64_t face_capacity,
                                        int64_t connection_capacity) {
  if (!out || !anchor || !width || n < 0 || (n > 0 && !d_generators)) return MV_ERR_ARG;
  out->n_cells = n;
  out->n_faces = 0;
  out->n_connections = 0;
  out->error_cell = -1;
  if (n > NMAX) return MV_ERR_CAPACITY;  // beyond the fixed scratch of this entry point
  mv_options o;
  mv_options_default(&o);
  if (opts_in) o = *opts_in;
  if (o.precision != MV_PRECISION_FP64 && o.precision != MV_PRECISION_FILTERED) return MV_ERR_ARG;
  if (o.face_mode != MV_FACES_OWNED && o.face_mode != MV_FACES_ALL) return MV_ERR_ARG;
  const bool csr = o.face_mode == MV_FACES_OWNED;
  if (n > 0 && (!out->cell_volume || !out->cell_centroid || !out->cell_safety_radius ||
                !out->face_left || !out->face_right || !out->face_area || !out->face_centroid ||
                !out->face_normal || !out->face_shift_code))
    return MV_ERR_ARG;
  if (n > 0 && csr && (!out->cell_face_offset || !out->cell_face_count || !out->cell_face_connections))
    return MV_ERR_ARG;
  Setup s;
  int rc = make_setup(n, anchor, width, dimensionality, periodic, o, &s);
  if (rc) return rc;
  const int64_t ncell = (int64_t)s.G[0] * s.G[1] * s.G[2];
  if (ncell > CELLMAX) return MV_ERR_CAPACITY;  // grid finer than the fixed scratch allows
  int dev = 0;
  NA_CUDA(cudaGetDevice(&dev));
  DeviceSetup* ds = nullptr;
  rc = device_setup(dev, &ds);
  if (rc) return rc;
  if (n == 0) return MV_OK;
  cudaStream_t st = (cudaStream_t)o.stream;
  unsigned char* B = ds->base;
  DevCounters* C = at<DevCounters>(B, O_COUNTERS);
  const int ni = (int)n;

  // clear what must start at zero (the array keeps the previous call's contents)
  NA_CUDA(cudaMemsetAsync(C, 0, sizeof(DevCounters), st));
  // the failing cell is a minimum over the failing cells: start above every index
  NA_CUDA(cudaMemsetAsync(C->status + STATUS_CELL, 0x7f, sizeof(int32_t), st));
  NA_CUDA(cudaMemsetAsync(C->ext_keys, 0xff, 3 * sizeof(unsigned long long), st));
  NA_CUDA(cudaMemsetAsync(B + O_CCOUNT, 0, 4 * (ncell + 1), st));
  NA_CUDA(cudaMemsetAsync(B + O_CFILL, 0, 4 * (ncell + 1), st));

  launch_prep(d_generators, ni, s.dim, at<double>(B, O_GEN), C->ext_keys, C->ext, &C->bad_input, st);
  launch_grid(at<double>(B, O_GEN), ni, s.G, s.anchor, s.ginv, at<int32_t>(B, O_CID),
              at<int32_t>(B, O_CCOUNT), at<int32_t>(B, O_CSTART), at<int32_t>(B, O_CFILL),
              at<double>(B, O_SX), at<double>(B, O_SY), at<double>(B, O_SZ), at<int32_t>(B, O_SID),
              at<long long>(B, O_SCAN), st);

  Job J;
  std::memset(&J, 0, sizeof(J));
  J.gen = at<double>(B, O_GEN);
  J.sx = at<double>(B, O_SX);
  J.sy = at<double>(B, O_SY);
  J.sz = at<double>(B, O_SZ);
  J.sid = at<int32_t>(B, O_SID);
  J.cell_start = at<int32_t>(B, O_CSTART);
  J.mask = d_mask;
  J.n = ni;
  J.dim = s.dim;
  J.periodic = s.periodic;
  J.face_mode = o.face_mode;
  J.precision = o.precision;
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
  J.ext = C->ext;
  J.R0 = s.R0;
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
  J.volume = out->cell_volume;
  J.centroid = out->cell_centroid;
  J.safety_radius = out->cell_safety_radius;
  J.face_count = at<int32_t>(B, O_FCOUNT);
  J.stage_off = at<int64_t>(B, O_STOFF);
  J.f_left = at<int32_t>(B, O_STLEFT);
  J.f_right = at<int32_t>(B, O_STRIGHT);
  J.f_area = at<double>(B, O_STAREA);
  J.f_centroid = at<double>(B, O_STCEN);
  J.f_normal = at<double>(B, O_STNRM);
  J.f_code = at<uint8_t>(B, O_STCODE);
  J.face_counter = &C->face_counter;
  J.face_cap = FACEMAX;
  J.order = nullptr;
  J.n_order = ni;
  J.work_counter = &C->work[0];
  J.ovf_list = at<int32_t>(B, O_OVFA);
  J.ovf_count = &C->ovf_count[0];
  J.status = C->status;
  J.stats = C->stats;
  const int pi = o.precision == MV_PRECISION_FILTERED ? 1 : 0;
  NA_CUDA(launch_cells(J, false, ds->sm_count * std::max(1, ds->bps_fast[pi]), st,
                       JobTable{nullptr, nullptr, 0}));
  DevCounters hc;
  NA_CUDA(cudaMemcpyAsync(&hc, C, sizeof(DevCounters), cudaMemcpyDeviceToHost, st));
  NA_CUDA(cudaStreamSynchronize(st));
  if (hc.bad_input) return MV_ERR_ARG;
  if (hc.ovf_count[0] > 0 && !hc.status[STATUS_CODE] && !hc.status[STATUS_FACE_OVERFLOW]) {
    Job L = J;
    L.order = at<int32_t>(B, O_OVFA);
    L.n_order = (int32_t)hc.ovf_count[0];
    L.work_counter = &C->work[1];
    L.ovf_list = at<int32_t>(B, O_OVFB);
    L.ovf_count = &C->ovf_count[1];
    // one warp per block: block b stages its big shells in slot b
    L.big = reinterpret_cast<char*>(B + O_BIG);
    const int blocks = std::min<int>(NA_BIG_SLOTS, L.n_order);
    NA_CUDA(launch_cells(L, true, blocks, st, JobTable{nullptr, nullptr, 0}));
    NA_CUDA(cudaMemcpyAsync(&hc, C, sizeof(DevCounters), cudaMemcpyDeviceToHost, st));
    NA_CUDA(cudaStreamSynchronize(st));
  }
  if (hc.status[STATUS_CODE]) {
    out->error_cell = hc.status[STATUS_CELL];
    return hc.status[STATUS_CODE];
  }
  // the faces the build asked for (also when they outgrew the staging scratch)
  const int64_t F = (int64_t)hc.face_counter;
  out->n_faces = F;
  if (hc.ovf_count[1] > 0 || hc.status[STATUS_FACE_OVERFLOW]) return MV_ERR_CAPACITY;
  if (F > face_capacity) return MV_ERR_CAPACITY;

  // faces in the reference's order, into the caller's arrays
  scan_i32_to_i64(at<int32_t>(B, O_FCOUNT), n, at<int64_t>(B, O_FOFF), at<long long>(B, O_SCAN), st);
  FaceArrays stage{at<int32_t>(B, O_STLEFT), at<int32_t>(B, O_STRIGHT), at<double>(B, O_STAREA),
                   at<double>(B, O_STCEN), at<double>(B, O_STNRM), at<uint8_t>(B, O_STCODE)};
  FaceArrays fin{out->face_left, out->face_right, out->face_area,
                 out->face_centroid, out->face_normal, out->face_shift_code};
  launch_reorder(stage, F, at<int64_t>(B, O_STOFF), at<int64_t>(B, O_FOFF), fin, st);
  if (csr) {
    NA_CUDA(cudaMemsetAsync(B + O_INCNT, 0, 4 * n, st));
    NA_CUDA(cudaMemsetAsync(B + O_CURSOR, 0, 4 * n, st));
    launch_csr_counts(fin, F, at<int32_t>(B, O_FCOUNT), ni, at<int32_t>(B, O_INCNT),
                      out->cell_face_count, st);
    scan_i32_to_i64(out->cell_face_count, n, at<int64_t>(B, O_CONNOFF), at<long long>(B, O_SCAN), st);
    int64_t Cn = 0;
    NA_CUDA(cudaMemcpyAsync(&Cn, at<int64_t>(B, O_CONNOFF) + n, 8, cudaMemcpyDeviceToHost, st));
    NA_CUDA(cudaStreamSynchronize(st));
    out->n_connections = Cn;
    if (Cn > connection_capacity) return MV_ERR_CAPACITY;
    launch_csr_fill(fin, F, at<int64_t>(B, O_FOFF), at<int64_t>(B, O_CONNOFF), at<int32_t>(B, O_INCNT),
                    at<int32_t>(B, O_CURSOR), ni, out->cell_face_connections, st);
    NA_CUDA(cudaMemcpyAsync(out->cell_face_offset, at<int64_t>(B, O_CONNOFF), 8 * n,
                            cudaMemcpyDeviceToDevice, st));
  }
  NA_CUDA(cudaGetLastError());
  NA_CUDA(cudaStreamSynchronize(st));
  return MV_OK;
}
