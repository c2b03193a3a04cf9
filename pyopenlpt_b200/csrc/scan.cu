// Device-wide exclusive scan (three-phase: tile scan, scan of tile sums, add) and
// the CSR builder declared in olpt_scan.cuh.
#include "olpt_scan.cuh"

namespace olpt {
namespace {


constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;  // per thread per block tile
constexpr int kScanTile = kScanThreads * kScanItems;

// Phase 1: per-tile exclusive scan in place; tile totals to `sums`.
__global__ void scan_tiles_kernel(const int* in, int n, int* out, int* sums) {
  __shared__ int warp_tot[32];
  const int base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
  int v[kScanItems];
  int t = 0;
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) {
    v[j] = (base + j < n) ? in[base + j] : 0;
    t += v[j];
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int incl = t;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) warp_tot[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    int w = warp_tot[lane];
    int wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += y;
    }
    warp_tot[lane] = wi - w;
    if (lane == 31) sums[blockIdx.x] = wi;
  }
  __syncthreads();
  int run = warp_tot[wid] + incl - t;
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) {
    if (base + j < n) out[base + j] = run;
    run += v[j];
  }
}

// Phase 2: exclusive scan of tile sums (n_tiles <= kScanTile), single CTA; total to sums[n_tiles].
__global__ void scan_sums_kernel(int* sums, int n_tiles) {
  __shared__ int buf[kScanTile + 1];
  for (int i = threadIdx.x; i < n_tiles; i += blockDim.x) buf[i] = sums[i];
  __syncthreads();
  if (threadIdx.x == 0) {
    int acc = 0;
    for (int i = 0; i < n_tiles; ++i) {
      int t = buf[i];
      buf[i] = acc;
      acc += t;
    }
    buf[n_tiles] = acc;
  }
  __syncthreads();
  for (int i = threadIdx.x; i <= n_tiles; i += blockDim.x) sums[i] = buf[i];
}

// Phase 3: add tile offsets; out[n] = total.
__global__ void scan_add_kernel(int* out, int n, const int* sums, int n_tiles) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] += sums[i / kScanTile];
  if (i == 0) out[n] = sums[n_tiles];
}

}  // namespace

void exclusive_scan(const int* in, int n, int* out, DevBuf& tmp, cudaStream_t s) {
  const int n_tiles = (n + kScanTile - 1) / kScanTile;
  OLPT_REQUIRE(n_tiles <= kScanTile, OLPT_ERR_UNSUPPORTED, "scan longer than 16M entries");
  tmp.ensure((n_tiles + 1) * sizeof(int), s);
  if (n > 0) {
    scan_tiles_kernel<<<OLPT_G(n_tiles), kScanThreads, 0, s>>>(in, n, out, tmp.as<int>());
    scan_sums_kernel<<<OLPT_G(1), 1024, 0, s>>>(tmp.as<int>(), n_tiles);
    scan_add_kernel<<<OLPT_G((n + 255) / 256), 256, 0, s>>>(out, n, tmp.as<int>(), n_tiles);
  } else {
    OLPT_CUDA(cudaMemsetAsync(out, 0, sizeof(int), s));
  }
  OLPT_CUDA(cudaGetLastError());
}

namespace {

// CSR scatter: items with key >= 0 go to bucket `key`; `cursor` must be zeroed.
__global__ void csr_scatter_kernel(const int* key, int n, const int* start, int* cursor,
                                   int* items) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int k = key[i];
  if (k < 0) return;
  items[start[k] + atomicAdd(&cursor[k], 1)] = i;
}

// Ascending item order inside every bucket (makes the CSR deterministic).
__global__ void csr_sort_kernel(const int* start, int n_buckets, int* items) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_buckets) return;
  const int b = start[c], e = start[c + 1];
  for (int i = b + 1; i < e; ++i) {
    const int v = items[i];
    int j = i - 1;
    while (j >= b && items[j] > v) {
      items[j + 1] = items[j];
      --j;
    }
    items[j + 1] = v;
  }
}

__global__ void csr_count_kernel(const int* key, int n, int* counts) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int k = key[i];
  if (k >= 0) atomicAdd(&counts[k], 1);
}

}  // namespace

void Csr::build(const int* key, int n, int n_buckets, cudaStream_t s, bool sort_buckets) {
    start.ensure((n_buckets + 1) * sizeof(int), s);
    cursor.ensure((n_buckets + 1) * sizeof(int), s);
    items.ensure((n + 1) * sizeof(int), s);
    OLPT_CUDA(cudaMemsetAsync(cursor.p, 0, n_buckets * sizeof(int), s));
    if (n > 0) csr_count_kernel<<<OLPT_G((n + 255) / 256), 256, 0, s>>>(key, n, cursor.as<int>());
    exclusive_scan(cursor.as<int>(), n_buckets, start.as<int>(), tmp, s);
    OLPT_CUDA(cudaMemsetAsync(cursor.p, 0, n_buckets * sizeof(int), s));
    if (n > 0) {
      csr_scatter_kernel<<<OLPT_G((n + 255) / 256), 256, 0, s>>>(key, n, start.as<int>(), cursor.as<int>(),
                                                         items.as<int>());
      if (sort_buckets)
        csr_sort_kernel<<<OLPT_G((n_buckets + 255) / 256), 256, 0, s>>>(start.as<int>(), n_buckets,
                                                                items.as<int>());
    }
    OLPT_CUDA(cudaGetLastError());
}

}  // namespace olpt
