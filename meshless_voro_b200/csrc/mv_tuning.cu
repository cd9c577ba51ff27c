// mv_tuning.cu -- the launch-tuning table (no counterpart in the reference crate).
//
// A build takes the parameters that its options leave at their defaults (pipeline
// MV_PIPELINE_AUTO, initial_radius 0, points_per_grid_cell 0, chunk_cells 0) from the
// table entry of its dimensionality and size band.  The built-in table
// (mv_tuning_table.h) is what the project's autotuner (meshless_voro_b200/autotune.py)
// measured on a B200; mv_tuning_set replaces it for the process.
#include <cstdint>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/mvgpu.h"
#include "mv_tuning_table.h"

namespace {

std::mutex g_tuning_mutex;
std::vector<mv_tuning_entry> g_tuning(kBuiltinTuning,
                                      kBuiltinTuning + sizeof(kBuiltinTuning) / sizeof(kBuiltinTuning[0]));

bool valid(const mv_tuning_entry& e) {
  return e.dimensionality >= 1 && e.dimensionality <= 3 &&
         (e.pipeline == MV_PIPELINE_STAGED || e.pipeline == MV_PIPELINE_FUSED) && e.n_min >= 0 &&
         e.n_max > e.n_min && e.initial_radius > 0.0 && e.initial_radius < 64.0 &&
         e.points_per_grid_cell > 0.0 && e.points_per_grid_cell < 1024.0 && e.chunk_cells > 0;
}

}  // namespace

namespace mv {

// The entry for a build of n generators in `dim` dimensions: the table's, or the
// library's fixed rule where no entry covers the band.
mv_tuning_entry tuned_params(int dim, int64_t n) {
  mv_tuning_entry d;
  std::memset(&d, 0, sizeof(d));
  d.dimensionality = dim;
  d.pipeline = n >= 65536 ? MV_PIPELINE_STAGED : MV_PIPELINE_FUSED;
  d.n_min = 0;
  d.n_max = INT64_MAX;
  d.initial_radius = dim == 3 ? 2.8 : (dim == 2 ? 2.4 : 2.2);
  d.points_per_grid_cell = 2.2;
  d.chunk_cells = 1 << 20;
  std::lock_guard<std::mutex> lock(g_tuning_mutex);
  for (const mv_tuning_entry& e : g_tuning)
    if (e.dimensionality == dim && n >= e.n_min && n < e.n_max) return e;
  return d;
}

}  // namespace mv

extern "C" int mv_tuning_set(const mv_tuning_entry* entries, int count) {
  if (count < 0 || (count > 0 && !entries)) return MV_ERR_ARG;
  for (int i = 0; i < count; i++)
    if (!valid(entries[i])) return MV_ERR_ARG;
  std::lock_guard<std::mutex> lock(g_tuning_mutex);
  if (count == 0)
    g_tuning.assign(kBuiltinTuning, kBuiltinTuning + sizeof(kBuiltinTuning) / sizeof(kBuiltinTuning[0]));
  else
    g_tuning.assign(entries, entries + count);
  return MV_OK;
}

extern "C" int mv_tuning_lookup(int dimensionality, int64_t n, mv_tuning_entry* out) {
  if (!out || dimensionality < 1 || dimensionality > 3 || n < 0) return MV_ERR_ARG;
  *out = mv::tuned_params(dimensionality, n);
  return MV_OK;
}

extern "C" int mv_tuning_count(void) {
  std::lock_guard<std::mutex> lock(g_tuning_mutex);
  return (int)g_tuning.size();
}
