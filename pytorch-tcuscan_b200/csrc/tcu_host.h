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
// SpMV products written as pre-split fp32 rows (64 bf16 hi then 64 bf16 lo
// per 64 products); prod holds roundup(nnz, 64) * 4 bytes.
// Full scan on the SIMT cores for small inputs (tcu_scan_small.cu); start
// plus the optional device start value as in the tensor-core scan.
tcu_status_t scan_small(const void* x, tcu_dtype_t dt, int64_t n, void* z, double start, void* ws, size_t ws_bytes,
                        cudaStream_t st, const void* start_dev, int start_dev_kind);
tcu_status_t spmv_products_split(const void* values, tcu_dtype_t dtype, const int32_t* cols, int64_t nnz,
                                 const void* x, int64_t x_len, void* prod, void* ws, void* stream);

}  // namespace tcu
