// Allocation-free sampler: amm_pick_sorted_noalloc (include/amm.h).
//
// The same draw as the context sampler (xorshift32 + mantissa uniform + inverse CDF, the
// reference's get_rand / pick_index, device_memory.h:506-545) followed by the ascending sort of
// the picks (the reference's CUB SortKeys, powerMethod_by_previous.cuh:63-70), for callers that
// may not allocate device memory at all: a host process that has handed the whole device to its
// own memory pool (any further cudaMalloc fails or breaks the pool's accounting), or a loop on a
// fixed latency budget in which an allocator call, which can synchronise the device, is not
// acceptable.  Such a caller cannot create an amm_ctx (its buffers are allocated), so this entry
// point takes the CDF and the xorshift states directly.
//
// Its only working memory is the file-scope array g_scratch below (1 MiB of multiplicities plus
// two 1 KiB tile tables): n is limited to kMaxColumns.  The multiplicity histogram must be zero
// for the draw; the call zeroes rows [0, n) itself as its first kernel, so nothing has to be
// zero on entry and a call that failed half-way leaves nothing behind that affects the next.
// The tile tables are rewritten by every call.  Because the array is shared by every call on a
// device, two calls that overlap in time (different streams, or different host threads without
// ordering) race on it and return garbage: serialise them.
//
// Launch sequence (stream-ordered on the caller's stream): clear -> draw -> tile sums ->
// expand.  One set-up per device resolves the array's address with cudaGetSymbolAddress; that
// first call on each device should come before any stream capture begins.

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "amm.h"
#include "amm_device.cuh"
#include "amm_internal.h"

namespace amm {
namespace {

constexpr int kMaxColumns = 1 << 18;                  // largest n (columns of the CDF)
constexpr int kTileThreads = 256;
constexpr int kTilePer = 4;                           // columns per thread
constexpr int kTile = kTileThreads * kTilePer;        // columns per tile (one CTA)
constexpr int kMaxTiles = kMaxColumns / kTile;        // 256
constexpr int kMaxDevices = 64;

struct NoAllocScratch {
  uint32_t count[kMaxColumns];  // multiplicity of each column among the c picks
  uint32_t tile_sum[kMaxTiles]; // picks per tile
  uint32_t tile_nz[kMaxTiles];  // distinct picked columns per tile
};

__device__ __align__(256) NoAllocScratch g_scratch;

__global__ void __launch_bounds__(kTileThreads) clear_kernel(NoAllocScratch* s, int n) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
    s->count[j] = 0u;
}

// First i in [0, n) with cdf[i] > target, else n-1: plain bisection (the reference's
// pick_index; the context sampler reaches the same index through a coarse table).
template <typename F>
__device__ __forceinline__ uint32_t first_above(const F* __restrict__ cdf, int n, F target) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(cdf + mid) <= target)
      lo = mid + 1;
    else
      hi = mid;
  }
  return static_cast<uint32_t>(lo < n ? lo : n - 1);
}

template <typename F>
__global__ void __launch_bounds__(kTileThreads) draw_kernel(NoAllocScratch* s,
                                                             const uint32_t* st_in,
                                                             uint32_t* st_out, int c,
                                                             const F* __restrict__ cdf, int n) {
  const F total = __ldg(cdf + n - 1);
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < c; k += gridDim.x * blockDim.x) {
    const uint32_t y = xorshift32(st_in[k]);
    st_out[k] = y;
    const float u = uniform_from(y);
    F target;
    if constexpr (sizeof(F) == 8)
      target = __dmul_rn(total, static_cast<double>(u));
    else
      target = __fmul_rn(total, u);
    atomicAdd(&s->count[first_above<F>(cdf, n, target)], 1u);
  }
}

// Per tile: number of picks and number of distinct picked columns.
__global__ void __launch_bounds__(kTileThreads) tile_kernel(NoAllocScratch* s, int n) {
  __shared__ uint32_t scan[40];
  const int j0 = blockIdx.x * kTile + threadIdx.x * kTilePer;
  uint32_t sum = 0, nz = 0;
#pragma unroll
  for (int e = 0; e < kTilePer; ++e) {
    const uint32_t v = j0 + e < n ? s->count[j0 + e] : 0u;
    sum += v;
    nz += v ? 1u : 0u;
  }
  uint32_t tot_sum, tot_nz;
  block_exclusive_scan(sum, scan, &tot_sum);
  block_exclusive_scan(nz, scan, &tot_nz);
  if (threadIdx.x == 0) {
    s->tile_sum[blockIdx.x] = tot_sum;
    s->tile_nz[blockIdx.x] = tot_nz;
  }
}

// Per tile: its offset in the sorted output (picks of the tiles before it), then each picked
// column j written count[j] times at its rank.  Tile 0 also writes the distinct count.
__global__ void __launch_bounds__(kTileThreads) expand_kernel(NoAllocScratch* s, int n,
                                                               uint32_t* out, int32_t* distinct) {
  __shared__ uint32_t scan[40];
  const int t = threadIdx.x;
  uint32_t before = 0;
  for (int k = t; k < (int)blockIdx.x; k += kTileThreads) before += s->tile_sum[k];
  uint32_t base;
  block_exclusive_scan(before, scan, &base);
  if (blockIdx.x == 0) {
    uint32_t nz = 0;
    for (int k = t; k < (int)gridDim.x; k += kTileThreads) nz += s->tile_nz[k];
    uint32_t total;
    block_exclusive_scan(nz, scan, &total);
    if (t == 0) *distinct = (int32_t)total;
  }
  const int j0 = blockIdx.x * kTile + t * kTilePer;
  uint32_t cnt[kTilePer];
  uint32_t sum = 0;
#pragma unroll
  for (int e = 0; e < kTilePer; ++e) {
    cnt[e] = j0 + e < n ? s->count[j0 + e] : 0u;
    sum += cnt[e];
  }
  uint32_t unused;
  uint32_t pos = base + block_exclusive_scan(sum, scan, &unused);
#pragma unroll
  for (int e = 0; e < kTilePer; ++e)
    for (uint32_t r = 0; r < cnt[e]; ++r) out[pos++] = (uint32_t)(j0 + e);
}

std::mutex g_setup_mutex;
NoAllocScratch* g_scratch_ptr[kMaxDevices] = {};

// Address of g_scratch on the current device, resolved once per device.
int scratch_for_current_device(NoAllocScratch** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return record_cuda_failure(e, "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) return AMM_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess) return record_cuda_failure(e, "cudaGetSymbolAddress(g_scratch)");
    g_scratch_ptr[dev] = static_cast<NoAllocScratch*>(p);
  }
  *out = g_scratch_ptr[dev];
  return AMM_OK;
}

}  // namespace
}  // namespace amm

extern "C" int amm_pick_sorted_noalloc(const uint32_t* d_states_in, uint32_t* d_states_out,
                                       int64_t c, const void* d_cdf, int cdf_precision, int64_t n,
                                       uint32_t* d_idx_sorted, int32_t* d_distinct, void* stream) {
  using namespace amm;
  if (!d_states_in || !d_states_out || !d_cdf || !d_idx_sorted || !d_distinct)
    return AMM_ERR_INVALID_ARGUMENT;
  if (c < 1 || c > INT32_MAX || n < 1) return AMM_ERR_INVALID_ARGUMENT;
  if (cdf_precision != AMM_CDF_F64 && cdf_precision != AMM_CDF_F32)
    return AMM_ERR_INVALID_ARGUMENT;
  if (n > kMaxColumns) return AMM_ERR_UNSUPPORTED;  // beyond the fixed scratch array
  NoAllocScratch* s = nullptr;
  int rc = scratch_for_current_device(&s);
  if (rc) return rc;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const int ni = (int)n, ci = (int)c;
  const int tiles = (ni + kTile - 1) / kTile;
  int draw_blocks = (ci + kTileThreads - 1) / kTileThreads;
  if (draw_blocks > 4096) draw_blocks = 4096;
  clear_kernel<<<tiles, kTileThreads, 0, st>>>(s, ni);
  if (cdf_precision == AMM_CDF_F64)
    draw_kernel<double><<<draw_blocks, kTileThreads, 0, st>>>(
        s, d_states_in, d_states_out, ci, static_cast<const double*>(d_cdf), ni);
  else
    draw_kernel<float><<<draw_blocks, kTileThreads, 0, st>>>(
        s, d_states_in, d_states_out, ci, static_cast<const float*>(d_cdf), ni);
  tile_kernel<<<tiles, kTileThreads, 0, st>>>(s, ni);
  expand_kernel<<<tiles, kTileThreads, 0, st>>>(s, ni, d_idx_sorted, d_distinct);
  count_launch(4);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return record_cuda_failure(e, "amm_pick_sorted_noalloc launch");
  return AMM_OK;
}
