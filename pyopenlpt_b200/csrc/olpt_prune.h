// Device candidate ordering and prune (prune.cu); the sequential greedy
// (greedy_select, stereo_host.cpp) remains the fallback.
#pragma once
#include <cuda_runtime.h>

#include "olpt_ctx.cuh"

namespace olpt {

void radix_sort_device(DevBuf& key, DevBuf& val, DevBuf& key2, DevBuf& val2, DevBuf& hist,
                       DevBuf& scan_tmp, int n, int bits, cudaStream_t s);
bool sort_candidates_device(PruneWork& W, const int* ids, const double* e, const double* X, int M,
                            int n, int max_id, cudaStream_t s);
bool prune_order_device(PruneWork& W, const PruneView& pv, int M, int n, int64_t total_points,
                        int* G_out, cudaStream_t s);
bool greedy_device(PruneWork& W, int M, int G, int n, int64_t total_points, uint8_t* sel,
                   cudaStream_t s);

}  // namespace olpt
