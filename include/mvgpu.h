/* mvgpu.h -- C ABI of the B200 (sm_100a) meshless Voronoi cell-construction library.
 *
 * Drop-in boundary for the per-cell construction path of the Rust crate
 * meshless_voronoi 0.7.2.  Each entry point below names the reference interface it
 * replaces (file:line in the crate).  All functions are thread-safe per context; a
 * context must not be used by two host threads at once.
 *
 * Layouts follow the reference: generators are `&[DVec3]` (n x 3 doubles, 24-byte
 * stride); cells, faces and cell->face connections come out in the reference's
 * order (faces grouped by their left cell in cell order, inside a cell in clipping-
 * plane order; connections per cell in increasing face index, voronoi.rs:241-263).
 * Indices are int32 (a tessellation holds fewer than 2^31 generators and faces);
 * a Rust binding widens them to usize.
 */
#ifndef MVGPU_H
#define MVGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (the reference panics where these are returned) ---- */
enum {
  MV_OK = 0,
  MV_ERR_ARG = 1,          /* invalid argument                                        */
  MV_ERR_DEGENERATE = 2,   /* duplicate generators: convex_cell.rs:325-329, 342       */
  MV_ERR_RING = 3,         /* no ring extension found: convex_cell.rs:428             */
  MV_ERR_DET = 4,          /* singular 3-plane intersection: geometry.rs:70           */
  MV_ERR_CAPACITY = 5,     /* a cell outgrew the largest device capacity tier         */
  MV_ERR_CUDA = 6,         /* a CUDA runtime call failed                              */
  MV_ERR_NO_DEVICE = 7,    /* no usable CUDA device                                   */
  MV_ERR_OOM = 8           /* device or pinned-host allocation failed                 */
};

/* ---- predicate precision ---- */
enum {
  MV_PRECISION_FP64 = 0,      /* every clip test in f64, as the reference            */
  MV_PRECISION_FILTERED = 1   /* f32 test under a proven bound, f64 + exact fallback */
};

/* ---- which faces a build emits ---- */
enum {
  MV_FACES_OWNED = 0,  /* Voronoi::build and compute_face_integrals_sym: one per face */
  MV_FACES_ALL = 1     /* compute_face_integrals: every face of every built cell      */
};

/* ---- dimensionality (voronoi.rs:31-40) ---- */
enum { MV_DIM_1 = 1, MV_DIM_2 = 2, MV_DIM_3 = 3 };

/* ---- how the cells are built (results are identical either way) ---- */
enum {
  MV_PIPELINE_AUTO = 0,    /* staged for large builds, fused for small ones          */
  MV_PIPELINE_STAGED = 1,  /* per chunk: shell, clip and integral kernels; cells that
                              need more than the first neighbour shell are rebuilt by
                              the fused kernel                                        */
  MV_PIPELINE_FUSED = 2    /* one kernel builds each cell from start to finish        */
};

typedef struct mv_options {
  int precision;                 /* MV_PRECISION_*                                   */
  int face_mode;                 /* MV_FACES_*                                       */
  double points_per_grid_cell;   /* 0: library default                               */
  double initial_radius;         /* first neighbour shell, in mean spacings; 0: default */
  void* stream;                  /* cudaStream_t to run on; NULL: the context stream */
  int pipeline;                  /* MV_PIPELINE_*                                    */
  int chunk_cells;               /* staged pipeline: cells per chunk; 0: default     */
} mv_options;

/* Per-build counters (escalations and retries). */
typedef struct mv_build_stats {
  int64_t cells_built;           /* active cells constructed                         */
  int64_t neighbours_clipped;    /* half-spaces tested against a cell                */
  int64_t planes_added;          /* half-spaces that removed at least one vertex     */
  int64_t f32_undecided;         /* filtered mode: f32 tests that fell back to f64   */
  int64_t exact_tests;           /* exact integer in-sphere evaluations              */
  int64_t extra_shells;          /* neighbour-shell expansions beyond the first      */
  int64_t overflow_cells;        /* cells re-run in the large capacity tier          */
  int64_t serial_rings;          /* rings rebuilt by the serial fallback             */
  int64_t staged_retries;        /* staged pipeline: cells rebuilt by the fused kernel
                                  * (those neither staged round closed)              */
  int64_t device_bytes;          /* device workspace held by the context             */
  int64_t kernel_launches;       /* library kernels launched by the build            */
  double ms_grid;                /* device time: generator prep + uniform grid       */
  double ms_cells;               /* device time: cell construction kernels           */
  double ms_finalize;            /* device time: face ordering + cell->face CSR      */
  double ms_shell;               /* staged pipeline, within ms_cells: shell kernels  */
  double ms_clip;                /*   clip kernels                                   */
  double ms_integrate;           /*   integral kernels                               */
  double ms_retry;               /*   fused kernel on the retried cells              */
  int64_t staged_wide;           /* staged pipeline: cells the first round left to   *
                                  * the wide (long-list) round                       */
} mv_build_stats;

/* Device-resident result of a build.  Pointers are owned by the context and stay
 * valid until the next build on it or mv_context_destroy.  Arrays are indexed by
 * original generator index; inactive cells of a partial build hold zeros. */
typedef struct mv_device_voronoi {
  int64_t n_cells, n_faces, n_connections;
  double* cell_volume;        /* [n]                                                   */
  double* cell_centroid;      /* [n][3]                                                */
  double* cell_safety_radius; /* [n]                                                   */
  int64_t* cell_face_offset;  /* [n]  offset into cell_face_connections                */
  int32_t* cell_face_count;   /* [n]                                                   */
  int32_t* face_left;         /* [F]                                                   */
  int32_t* face_right;        /* [F]  -1: boundary face (right() == None)              */
  double* face_area;          /* [F]                                                   */
  double* face_centroid;      /* [F][3]                                                */
  double* face_normal;        /* [F][3] clipping-plane normal, towards the left cell   */
  uint8_t* face_shift_code;   /* [F]  13: no shift; else (mx+1)+3(my+1)+9(mz+1)        */
  int32_t* cell_face_connections; /* [C]                                               */
  int64_t error_cell;         /* first failing cell for error statuses, else -1        */
} mv_device_voronoi;

/* Host result (same arrays, host memory).  VoronoiCell::loc() is the generator with
 * unused dims zeroed for built cells and 0 for inactive ones (voronoi_cell.rs:107);
 * VoronoiFace::shift() is mv_shift_from_code(face_shift_code[f]). */
typedef struct mv_voronoi {
  int64_t n_cells, n_faces, n_connections;
  int dimensionality, periodic;
  double anchor[3], width[3];   /* normalised simulation volume (voronoi.rs:200-210)  */
  double* cell_volume;
  double* cell_centroid;
  double* cell_safety_radius;
  int64_t* cell_face_offset;
  int32_t* cell_face_count;
  int32_t* face_left;
  int32_t* face_right;
  double* face_area;
  double* face_centroid;
  double* face_normal;
  uint8_t* face_shift_code;
  int32_t* cell_face_connections;
  int64_t error_cell;           /* first failing cell for error statuses, else -1     */
  void* _owner;                 /* internal                                           */
} mv_voronoi;

typedef struct mv_context mv_context;

/* Default options: filtered precision, owned faces, context stream. */
void mv_options_default(mv_options* opts);

/* Human-readable message for a status code (never NULL). */
const char* mv_strerror(int status);

/* Library version string. */
const char* mv_version(void);

/* A context owns a CUDA stream, the device workspace (grown on demand and reused)
 * and a pinned host arena for results.  device < 0 selects the current device. */
int mv_context_create(int device, mv_context** ctx);
void mv_context_destroy(mv_context* ctx);

/* Counters of the last build on the context. */
int mv_context_last_stats(const mv_context* ctx, mv_build_stats* out);

/* Replaces Voronoi::build (voronoi.rs:151-159) and Voronoi::build_partial
 * (voronoi.rs:181-190) with device-resident inputs and outputs.
 * d_generators: device [n][3] doubles; d_mask: device [n] bytes (nonzero == true) or
 * NULL for a full build.  Returns when the result is complete on the device. */
int mv_context_build_device(mv_context* ctx, const double* d_generators, const uint8_t* d_mask,
                            int64_t n, const double anchor[3], const double width[3],
                            int dimensionality, int periodic, const mv_options* opts,
                            mv_device_voronoi* out);

/* Same as mv_context_build_device with host inputs; the result is copied into the
 * context's pinned host arena (valid until the next build on the context).  *out
 * is owned by the context: do not pass it to mv_voronoi_free.  Builds with host
 * buffers (this call, mv_context_build_cells and mv_context_build_batch) on one
 * device run their GPU phase one at a time and copy their results back outside it:
 * with one context per host thread, one build's result copy overlaps the next
 * build's kernels. */
int mv_context_build(mv_context* ctx, const double* generators, const uint8_t* mask, int64_t n,
                     const double anchor[3], const double width[3], int dimensionality,
                     int periodic, const mv_options* opts, mv_voronoi** out);

/* Stand-alone Voronoi::build (voronoi.rs:151-159): host in, host out, on the current
 * device with a temporary context.  Free the result with mv_voronoi_free. */
int mv_voronoi_build(const double* generators, int64_t n, const double anchor[3],
                     const double width[3], int dimensionality, int periodic,
                     const mv_options* opts, mv_voronoi** out);

/* Stand-alone Voronoi::build_partial (voronoi.rs:181-190). */
int mv_voronoi_build_partial(const double* generators, const uint8_t* mask, int64_t n,
                             const double anchor[3], const double width[3], int dimensionality,
                             int periodic, const mv_options* opts, mv_voronoi** out);

void mv_voronoi_free(mv_voronoi* v);

/* ---- the convex cells themselves (VoronoiIntegrator, voronoi.rs:527-828) ----
 *
 * A cells build returns, besides the Voronoi result, every built ConvexCell
 * (convex_cell.rs:53-60) as CSR arrays indexed by generator (inactive cells are
 * empty): its clipping planes and its vertices in the reference's order.  With
 * MV_CELLS_TETS it also returns the oriented tets that custom integrals consume
 * (CellIntegral::collect(v0, v1, v2, gen), integrals.rs:24-36; the generator is every
 * tet's apex), in the order compute_cell_integral / compute_face_integrals feed them
 * (convex_cell.rs:583-664): per vertex the six tets of DecompositionWithoutFaces, or,
 * with MV_CELLS_WITH_FACES, per face the fan of DecompositionWithFaces
 * (convex_cell.rs:89-129).  MV_CELLS_WITH_FACES also returns the faces of
 * ConvexCell::with_faces (convex_cell.rs:461-543): the planes holding at least one
 * vertex, in plane order, each with its vertex indices sorted by sort_face_vertices.
 * with_faces is 3D only: MV_CELLS_WITH_FACES in 1D or 2D returns MV_ERR_ARG (the
 * reference panics).  Plane and vertex indices are local to their cell. */
enum { MV_CELLS_TETS = 1, MV_CELLS_WITH_FACES = 2 };

typedef struct mv_cells {
  int64_t n_cells, n_planes, n_vertices, n_tets, n_faces, n_face_vertices;
  int64_t* cell_plane_offset;   /* [n + 1]                                            */
  double* plane_normal;         /* [P][3] HalfSpace normal (half_space.rs:9-19)       */
  double* plane_point;          /* [P][3] HalfSpace point p                           */
  int32_t* plane_right;         /* [P]    right generator, -1: boundary plane         */
  uint8_t* plane_shift_code;    /* [P]    13: no shift, see mv_shift_from_code        */
  int64_t* cell_vertex_offset;  /* [n + 1]                                            */
  double* vertex_loc;           /* [V][3] in the reference's vertex order             */
  int32_t* vertex_dual;         /* [V][3] the three planes meeting at the vertex      */
  int64_t* cell_tet_offset;     /* [n + 1]  (MV_CELLS_TETS)                           */
  double* tet_vertices;         /* [T][3][3] v0, v1, v2                               */
  int32_t* tet_plane;           /* [T]    the plane of the tet's base face            */
  int64_t* cell_face_offset;    /* [n + 1]  (MV_CELLS_WITH_FACES)                     */
  int32_t* face_plane;          /* [Fc]   the face's plane                            */
  int64_t* face_vertex_offset;  /* [Fc + 1] into face_vertices                        */
  int32_t* face_vertices;       /* [sum]  vertex indices, counter-clockwise           */
} mv_cells;

/* Cells build with device inputs: the Voronoi result as mv_context_build_device and the
 * cells as device pointers owned by the context (valid until its next build). */
int mv_context_build_cells_device(mv_context* ctx, const double* d_generators,
                                  const uint8_t* d_mask, int64_t n, const double anchor[3],
                                  const double width[3], int dimensionality, int periodic,
                                  const mv_options* opts, int cells_flags,
                                  mv_device_voronoi* voronoi, mv_cells* cells);

/* Cells build with host inputs: both results copied to the context's pinned host arena
 * (valid until the next build on the context; owned by the context). */
int mv_context_build_cells(mv_context* ctx, const double* generators, const uint8_t* mask,
                           int64_t n, const double anchor[3], const double width[3],
                           int dimensionality, int periodic, const mv_options* opts,
                           int cells_flags, mv_voronoi** voronoi, mv_cells** cells);

/* ---- batches: many tessellations in one build ----
 *
 * The reference builds one tessellation per call (Voronoi::build, voronoi.rs:151-238);
 * a caller with many independent tessellations (uneven sizes, mixed dimensionality,
 * periodic and rectangular, full and partial) calls it in a loop.  A batch build does
 * them together: one grid build, one pass of the cell kernels over all cells (each
 * cell finds its tessellation), one finalize, so the launch count does not grow with
 * the number of tessellations and small tessellations share the GPU.  Each
 * tessellation's result is exactly what mv_context_build_device returns for it alone.
 *
 * Inputs are concatenated: tessellation j's generators are the rows
 * [sum_{i<j} n_i, sum_{i<=j} n_i) of one [sum n][3] array (and of one mask array,
 * used for the tessellations with has_mask set). */
typedef struct mv_job {
  int64_t n;                 /* generators of the tessellation                        */
  double anchor[3];          /* simulation box, as Voronoi::build's anchor / width    */
  double width[3];
  int32_t dimensionality;    /* 1, 2 or 3                                             */
  int32_t periodic;
  int32_t has_mask;          /* build_partial: the tessellation's mask rows apply     */
  int32_t reserved;
} mv_job;

/* Result of a batch: the tessellations' results concatenated, each in the reference's
 * own indexing (cell and face indices local to the tessellation; cell_face_offset
 * relative to the tessellation's first connection).  Tessellation j owns cells
 * [job_cell_offset[j], job_cell_offset[j+1]), faces [job_face_offset[j], ...) and
 * connections [job_connection_offset[j], ...).  The offset arrays are host memory;
 * the other arrays are device memory for mv_context_build_batch_device and pinned
 * host memory for mv_context_build_batch.  All are owned by the context and valid
 * until its next build.  On an error status error_job / error_cell name the first
 * failing tessellation and its cell. */
typedef struct mv_batch_voronoi {
  int64_t n_jobs, n_cells, n_faces, n_connections;
  const int64_t* job_cell_offset;        /* [n_jobs + 1] */
  const int64_t* job_face_offset;        /* [n_jobs + 1] */
  const int64_t* job_connection_offset;  /* [n_jobs + 1] */
  double* cell_volume;
  double* cell_centroid;
  double* cell_safety_radius;
  int64_t* cell_face_offset;
  int32_t* cell_face_count;
  int32_t* face_left;
  int32_t* face_right;
  double* face_area;
  double* face_centroid;
  double* face_normal;
  uint8_t* face_shift_code;
  int32_t* cell_face_connections;
  int64_t error_job, error_cell;
} mv_batch_voronoi;

/* Batch build from device inputs (d_mask may be NULL when no job has has_mask). */
int mv_context_build_batch_device(mv_context* ctx, const double* d_generators, const uint8_t* d_mask,
                                  const mv_job* jobs, int64_t n_jobs, const mv_options* opts,
                                  mv_batch_voronoi* out);

/* Batch build from host inputs, results copied to the context's pinned host arena. */
int mv_context_build_batch(mv_context* ctx, const double* generators, const uint8_t* mask,
                           const mv_job* jobs, int64_t n_jobs, const mv_options* opts,
                           mv_batch_voronoi* out);

/* ---- launch tuning (no counterpart in the reference crate) ----
 *
 * The reference builds every cell the same way (voronoi.rs:265-315); this library has
 * launch parameters whose best values depend on the dimensionality and the size of a
 * build: the pipeline, the first neighbour shell's radius (initial_radius, in mean
 * generator spacings: how many neighbours are set up first), the uniform grid's
 * resolution (points_per_grid_cell) and the staged pipeline's chunk.  The library's
 * autotuner (meshless_voro_b200/autotune.py) measures them on a B200 per
 * dimensionality and size band; its table is built into the library.  A build takes
 * every parameter that its mv_options leave at the default (MV_PIPELINE_AUTO, 0) from
 * the entry whose band [n_min, n_max) holds its generator count.  Results never depend
 * on these parameters, only the time does. */
typedef struct mv_tuning_entry {
  int32_t dimensionality;        /* 1, 2 or 3                                        */
  int32_t pipeline;              /* MV_PIPELINE_STAGED or MV_PIPELINE_FUSED          */
  int64_t n_min, n_max;          /* generator counts n_min <= n < n_max              */
  double initial_radius;         /* first neighbour shell, in mean spacings          */
  double points_per_grid_cell;   /* uniform grid resolution                          */
  int32_t chunk_cells;           /* staged pipeline: cells per chunk                 */
  int32_t reserved;
} mv_tuning_entry;

/* Replaces the process-wide table (count == 0: back to the built-in one); returns
 * MV_ERR_ARG for an invalid entry (and keeps the table). */
int mv_tuning_set(const mv_tuning_entry* entries, int count);

/* The entry a build of n generators in `dimensionality` dimensions uses. */
int mv_tuning_lookup(int dimensionality, int64_t n, mv_tuning_entry* out);

/* Entries in the current table. */
int mv_tuning_count(void);

/* ---- build without allocating (no counterpart in the reference crate) ----
 *
 * For callers that cannot call cudaMalloc -- a host framework that has handed all
 * device memory to its own pool allocator, code that must not trigger the implicit
 * device synchronisation of cudaMalloc/cudaFree, or an embedding with a fixed memory
 * plan.  Same result as mv_context_build_device, on the current device, but every
 * scratch buffer lives in one fixed static device array inside the library, so the
 * call allocates nothing.  That array (about 51 MB) is held by every GPU that loads
 * the library until the process exits.
 *
 * Limits: at most MV_NOALLOC_MAX_GENERATORS generators (larger n returns
 * MV_ERR_CAPACITY without touching the GPU) and at most
 * MV_NOALLOC_FACES_PER_GENERATOR * MV_NOALLOC_MAX_GENERATORS staged faces (room for
 * MV_FACES_ALL on 3-D sets of the full size, about 15.5 faces per cell; a set that
 * needs more returns MV_ERR_CAPACITY with out->n_faces above that limit).
 *
 * The caller passes device inputs and fills `out` with device pointers sized for n
 * cells (cell_volume, cell_centroid, cell_safety_radius, and for MV_FACES_OWNED
 * cell_face_offset, cell_face_count), face_capacity faces (face_left ... face_shift_code)
 * and connection_capacity connections (cell_face_connections, MV_FACES_OWNED only).
 * On return out->n_faces / out->n_connections hold the sizes the build needed; when
 * they exceed the capacities the call returns MV_ERR_CAPACITY.  Runs on opts->stream
 * (NULL: the legacy default stream) and returns when the result is complete.  Cells
 * whose neighbour shells hold thousands of candidates (the surface of a dense clump)
 * are built by a few warps only, so such inputs run slower than in a context build.
 *
 * The first call on a device looks up the array's device address (once per device);
 * make that first call before any stream capture.  All calls share the array and it
 * keeps the previous call's contents (each call clears what must start at zero):
 * calls that overlap on the GPU -- from several host threads or streams -- race on it
 * and must be serialised by the caller. */
#define MV_NOALLOC_MAX_GENERATORS 32768
#define MV_NOALLOC_FACES_PER_GENERATOR 18
int mv_voronoi_build_noalloc(const double* d_generators, const uint8_t* d_mask, int64_t n,
                             const double anchor[3], const double width[3], int dimensionality,
                             int periodic, const mv_options* opts, mv_device_voronoi* out,
                             int64_t face_capacity, int64_t connection_capacity);

/* The reference's shift vector for a face shift code (rtree_nn.rs:27-33): component i
 * is m_i * width_i for m_i != 0 and -0.0 for m_i == 0, with (m_x, m_y, m_z) decoded
 * from code = (m_x+1) + 3(m_y+1) + 9(m_z+1).  Code 13 (no shift) gives all -0.0. */
void mv_shift_from_code(int code, const double width[3], double out[3]);

#ifdef __cplusplus
}
#endif

#endif /* MVGPU_H */
