// mv_tuning_table.h -- built-in launch tuning of libmvgpu (generated by
// `python -m meshless_voro_b200.autotune --write`; edit the JSON it reads from, not this).
// Source: meshless_voro_b200/tuning/b200.json
#pragma once
// {dimensionality, pipeline, n_min, n_max, initial_radius, points_per_grid_cell, chunk_cells, reserved}
static const mv_tuning_entry kBuiltinTuning[] = {
    {3, MV_PIPELINE_STAGED, 0, 8192, 2.8, 2.2, 1048576, 0},
    {3, MV_PIPELINE_STAGED, 8192, 32768, 2.8, 2.2, 1048576, 0},
    {3, MV_PIPELINE_STAGED, 32768, 131072, 2.8, 2.2, 1048576, 0},
    {3, MV_PIPELINE_STAGED, 131072, 524288, 2.8, 2.2, 1048576, 0},
    {3, MV_PIPELINE_STAGED, 524288, 2097152, 2.8, 2.2, 1048576, 0},
    {3, MV_PIPELINE_STAGED, 2097152, 8388608, 2.8, 2.2, 1048576, 0},
    {3, MV_PIPELINE_STAGED, 8388608, 4611686018427387904LL, 2.8, 2.2, 1048576, 0},
    {2, MV_PIPELINE_STAGED, 0, 8192, 2.4, 2.2, 1048576, 0},
    {2, MV_PIPELINE_STAGED, 8192, 32768, 3.2, 2.2, 1048576, 0},
    {2, MV_PIPELINE_STAGED, 32768, 131072, 3.2, 2.2, 1048576, 0},
    {2, MV_PIPELINE_STAGED, 131072, 524288, 3.2, 2.2, 1048576, 0},
    {2, MV_PIPELINE_STAGED, 524288, 2097152, 3.2, 2.2, 1048576, 0},
    {2, MV_PIPELINE_STAGED, 2097152, 4611686018427387904LL, 3.2, 2.2, 1048576, 0},
    {1, MV_PIPELINE_FUSED, 0, 65536, 2.2, 2.2, 1048576, 0},
    {1, MV_PIPELINE_STAGED, 65536, 4611686018427387904LL, 2.2, 2.2, 1048576, 0},
};
