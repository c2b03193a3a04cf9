// Device-wide exclusive prefix sum of int32 counts and a CSR builder
// (count -> scan -> scatter -> per-bucket ascending order), shared by the stereo
// cell grid, the shake tile bins and the 3D hash grid.  Implementation: scan.cu.
#pragma once
#include <cuda_runtime.h>

#include "olpt_ctx.cuh"

namespace olpt {

// out[0..n] = exclusive scan of in[0..n), out[n] = total.  `tmp` is scratch.
void exclusive_scan(const int* in, int n, int* out, DevBuf& tmp, cudaStream_t s);

}  // namespace olpt
