// tcu_host.h -- host-side helpers shared by the libtcuscan.so translation units.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "tcu_lookback.cuh"
#include "tcuscan.h"

namespace tcu {

tcu_status_t cuda_fail(cudaError_t e, const char* what);
uint64_t timeout_ns();
int sm_count();
int grid_ctas();
tcu_status_t make_map_2d(CUtensorMap* m, const void* base, CUtensorMapDataType dt, int elem, uint64_t cols,
                         uint64_t rows, uint32_t box_cols, uint32_t box_rows);
bool aligned16(const void* p);
int64_t ws_capacity(size_t bytes);
TileDesc* ws_descs(void* ws);
unsigned long long* ws_phase_counters(void* ws);

}  // namespace tcu
