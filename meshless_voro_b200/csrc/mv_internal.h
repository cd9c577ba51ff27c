// mv_internal.h -- structures shared by the kernels and the host orchestration.
#pragma once
#include <cmath>
#include <cstdint>

namespace mv {

// Per-build counters, accumulated on the device (see mv_build_stats in mvgpu.h).
enum StatSlot {
  ST_CELLS = 0,
  ST_NEIGHBOURS,
  ST_PLANES,
  ST_F32_UNDECIDED,
  ST_EXACT,
  ST_SHELLS,
  ST_OVERFLOW,
  ST_SERIAL_RING,
  ST_COUNT
};

// Device status words: [0] status code (first error wins), [1] failing cell (min),
// [2] set when the face staging buffer was too small, [3] set when the cell-record
// buffer of an export build was too small (the host grows the buffer and reruns).
enum { STATUS_CODE = 0, STATUS_CELL = 1, STATUS_FACE_OVERFLOW = 2, STATUS_REC_OVERFLOW = 3,
       STATUS_WORDS = 4 };

// Device counters of one build (one allocation, cleared before each build).
struct DevCounters {
  unsigned long long face_counter;
  unsigned long long stats[ST_COUNT];
  unsigned long long ext_keys[6];
  double ext[6];
  int32_t status[STATUS_WORDS];
  unsigned int work[4];       // work queues of the capacity tiers
  unsigned int ovf_count[4];  // overflow lists of the capacity tiers
  int32_t bad_input;
  int32_t pad[3];
  unsigned long long rec_counter;  // cell-record words allocated by an export build
};

// Face arrays (SoA; centroid and normal are [F][3]).
struct FaceArrays {
  int32_t* left;
  int32_t* right;
  double* area;
  double* centroid;
  double* normal;
  uint8_t* code;
};

// One tessellation, as seen by the cell kernel.
struct Job {
  // ---- generators ----
  const double* gen;        // [n][3] by original index, unused dims zeroed (generator.rs:13-24)
  const double* sx;         // grid-sorted SoA copies
  const double* sy;
  const double* sz;
  const int32_t* sid;       // sorted position -> original index
  const int32_t* cell_start;  // grid cell -> first sorted position, [ncell + 1]
  const uint8_t* mask;      // by original index, or nullptr (full build)
  int32_t n;
  int32_t dim;
  int32_t periodic;
  int32_t face_mode;        // MV_FACES_OWNED / MV_FACES_ALL
  int32_t precision;        // MV_PRECISION_*
  // ---- uniform grid ----
  int32_t G[3];
  double ga[3];             // grid anchor == normalised simulation anchor
  double gw[3];             // normalised simulation width (period of the images)
  double gh[3];             // cell size
  double ginv[3];           // 1 / cell size
  const double* ext;        // device [6]: min x,y,z, max x,y,z of the generators
  double geps[3];           // cell-box inflation against rounding of the cell index
  double R0;                // first neighbour-shell radius
  // second level in dense cells (all nullptr when no cell is dense): the generators of a
  // dense cell are sorted by the Morton key of their position inside the cell (fbits
  // bits per active axis, x lowest), so that every cell of the cell's implicit octree,
  // at any level 0..fbits, is a contiguous range of sorted positions
  const int32_t* dprefix;   // [ncell + 1] number of dense cells before each cell (row-major)
  const int32_t* cell_dense;  // [ncell] 1: dense
  const uint32_t* fkey;     // [n] Morton key by sorted position (meaningful in dense cells)
  int32_t fbits;
  double ppc_mean;          // generators per grid cell on average (first-radius scaling)
  // periodic image of shift code c = (mx+1) + 3(my+1) + 9(mz+1): the reference's query
  // offset s = (-m) w (rtree_nn.rs:86) and emitted shift -s (rtree_nn.rs:27-33)
  double qshift[27][3];
  double shift[27][3];
  // ---- simulation boundary (boundary.rs:14-47) ----
  double bn[6][3];
  double bp[6][3];
  double bd[6];
  double iloc_a[3];         // anchor - width of the (tripled) box
  double iloc_inv[3];       // 1 / (3 width)
  double xabs_max;          // max |coordinate| over generators (filter bound)
  // ---- outputs, by original index ----
  double* volume;
  double* centroid;         // [n][3]
  double* safety_radius;
  int32_t* face_count;      // faces emitted by the cell
  int64_t* stage_off;       // first staging slot of the cell's faces
  // ---- face staging (cells append in completion order) ----
  int32_t* f_left;
  int32_t* f_right;
  double* f_area;
  double* f_centroid;       // [cap][3]
  double* f_normal;         // [cap][3]
  uint8_t* f_code;
  unsigned long long* face_counter;
  int64_t face_cap;
  // ---- work distribution / retry queue ----
  const int32_t* order;     // sorted positions to process (retry / overflow pass), or nullptr
  int32_t n_order;          // number of positions to process
  unsigned int* work_counter;
  int32_t* ovf_list;        // cells that outgrew this capacity tier
  unsigned int* ovf_count;
  int32_t* status;          // [STATUS_WORDS]
  unsigned long long* stats;  // [ST_COUNT]
  // ---- cell records of an export build (nullptr otherwise): the fused kernel writes
  // the finished cells it builds, like the staged clip kernel ----
  double* rec;
  int64_t rec_cap;
  unsigned long long* rec_counter;
  int64_t* rec_off;         // by sorted position, -1: none
  // ---- per-warp staging slots of the fused kernel for shells larger than its shared
  // buffer (slot = global warp index), or nullptr ----
  char* big;
  // ---- batches: this tessellation's first position in the concatenated arrays of the
  // batch (0 for a single build); staged faces and error cells carry it, so that the
  // batch's finalize can find their tessellation ----
  int32_t id_base;
};

// The tessellations of a batch build.  Tessellation j holds the sorted positions (and
// input indices) [pos_base[j], pos_base[j + 1]) of the concatenated arrays; its Job
// addresses its own slices, so every index inside it is local, as in the reference.
struct JobTable {
  const Job* jobs;          // [njobs], device
  const int32_t* pos_base;  // [njobs + 1], device
  int32_t njobs;
};

// One chunk of the staged path: cells at processing positions [item0, item0 + nitems)
// go through the shell, clip and integral kernels.  The first round processes the
// cells in grid order; the second (wide) round takes the first round's retry list.
struct StageJob {
  int32_t item0;
  int32_t nitems;
  const int32_t* order;       // processing position -> sorted position, or nullptr (identity)
  int32_t cstride;            // candidate-list entries per cell
  uint32_t* cand;             // [nitems][cstride]: sorted position * 27 + shift code
  int32_t* info;              // [nitems]: count | exhausted << 30, 0: inactive, -1: retry
  double* rad;                // [nitems]: radius of the first shell (first_radius)
  int64_t* rec_off;           // [nitems]: word offset of the cell record, -1: none
  double* rec;                // cell records (planes, vertices) for the integral kernel
  int64_t rec_cap;            // record words available to the chunk
  unsigned long long* rec_counter;
  int32_t full_records;       // 1: full records (export builds), 0: compact (write_record)
  int32_t box;                // 1: the clip kernel decides box-corner band tests itself
  unsigned int* work;         // [3] work counters of the shell, clip and integral kernels
  int32_t* retry_list;        // positions the next round (wide round, fused kernel) takes
  unsigned int* retry_count;
  int32_t* fused_list;        // positions that go straight to the fused kernel (exact tests)
  unsigned int* fused_count;
};

// Grid of one tessellation of a batch (the batch grid kernels, mv_grid.cu).
struct BatchGrid {
  int G[3];
  int dim;
  double a[3], inv[3];
  int32_t cbase;  // first batch-wide grid cell of the tessellation
  int32_t pad;
};

// Normalised simulation volume, boundary planes (boundary.rs:14-47), uniform grid and
// first shell radius of one tessellation (mv_api.cu).
struct Setup {
  double anchor[3], width[3];
  int dim, periodic;
  int G[3];
  double gh[3], ginv[3], geps[3];
  double R0;
  double bn[6][3], bp[6][3], bd[6];
  double iloc_a[3], iloc_inv[3];
};

// Morton keys of the dense-cell octrees: FKEY_BITS bits in all, fkey_bits(dim) per
// active axis; bit (dim * b + i) of a key is bit b of the sub-cell index along axis i.
constexpr int FKEY_BITS = 30;
__host__ __device__ inline int fkey_bits(int dim) { return dim == 3 ? 10 : (dim == 2 ? 15 : 20); }
__host__ __device__ inline uint32_t spread2(uint32_t v) {  // 10 bits -> every third bit
  v &= 0x3ffu;
  v = (v | (v << 16)) & 0x030000ffu;
  v = (v | (v << 8)) & 0x0300f00fu;
  v = (v | (v << 4)) & 0x030c30c3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}
__host__ __device__ inline uint32_t spread1(uint32_t v) {  // 16 bits -> every other bit
  v &= 0xffffu;
  v = (v | (v << 8)) & 0x00ff00ffu;
  v = (v | (v << 4)) & 0x0f0f0f0fu;
  v = (v | (v << 2)) & 0x33333333u;
  v = (v | (v << 1)) & 0x55555555u;
  return v;
}
__host__ __device__ inline uint32_t morton(int dim, uint32_t x, uint32_t y, uint32_t z) {
  return dim == 3 ? (spread2(x) | (spread2(y) << 1) | (spread2(z) << 2))
                  : (dim == 2 ? (spread1(x) | (spread1(y) << 1)) : x);
}
// Sub-cell index (at the finest level) of coordinate g inside coarse cell c along one axis.
__host__ __device__ inline uint32_t fine_q(double g, double a, double inv, int c, int bits) {
  const double top = (double)((1u << bits) - 1u);
  double t = floor(((g - a) * inv - (double)c) * (double)(1u << bits));
  if (!(t >= 0.0)) t = 0.0;
  if (t > top) t = top;
  return (uint32_t)t;
}

}  // namespace mv

struct mv_options;
namespace mv {
int make_setup(int64_t n, const double* anchor, const double* width, int dim, int periodic,
               const mv_options& o, Setup* s);
}  // namespace mv
