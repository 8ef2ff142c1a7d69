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
// Launch sequence (stream-ordered on the caller's stream): clear -> draw -> tile prefix ->
// expand.  The expansion is parallel over the c output positions (each finds its tile and then
// its column by binary search), so a CDF that puts every pick on one column costs no more than
// a spread one.  Every call resolves the array's device address with cudaGetSymbolAddress for
// the current device (a lookup once the module is loaded; the first call on a device loads it,
// so that first call should come before any stream capture begins).

#include <cuda_runtime.h>

#include <cstdint>

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

// Per tile: number of picks and number of distinct picked columns; the multiplicities of the
// tile become their inclusive prefix within the tile (in place), the expansion's search table.
__global__ void __launch_bounds__(kTileThreads) tile_kernel(NoAllocScratch* s, int n) {
  __shared__ uint32_t scan[40];
  const int j0 = blockIdx.x * kTile + threadIdx.x * kTilePer;
  uint32_t cnt[kTilePer];
  uint32_t sum = 0, nz = 0;
#pragma unroll
  for (int e = 0; e < kTilePer; ++e) {
    cnt[e] = j0 + e < n ? s->count[j0 + e] : 0u;
    sum += cnt[e];
    nz += cnt[e] ? 1u : 0u;
  }
  uint32_t tot_sum, tot_nz;
  uint32_t run = block_exclusive_scan(sum, scan, &tot_sum);
  block_exclusive_scan(nz, scan, &tot_nz);
#pragma unroll
  for (int e = 0; e < kTilePer; ++e) {
    run += cnt[e];
    if (j0 + e < n) s->count[j0 + e] = run;
  }
  if (threadIdx.x == 0) {
    s->tile_sum[blockIdx.x] = tot_sum;
    s->tile_nz[blockIdx.x] = tot_nz;
  }
}

// Output position p of the sorted picks (0 <= p < c) holds the column j whose picks cover it:
// its tile is the last one whose first position is <= p (the exclusive prefix of the tile
// totals, in shared memory), and within the tile the first column whose inclusive prefix
// exceeds p's rank in the tile.  Block 0 also writes the number of distinct columns.
__global__ void __launch_bounds__(kTileThreads) expand_kernel(NoAllocScratch* s, int n, int tiles,
                                                               int c, uint32_t* out,
                                                               int32_t* distinct) {
  __shared__ uint32_t first[kMaxTiles + 1];
  __shared__ uint32_t scan[40];
  const int t = threadIdx.x;
  // exclusive prefix of the tile totals: kMaxTiles / kTileThreads tiles per thread, in order
  constexpr int kPer = kMaxTiles / kTileThreads;
  uint32_t v[kPer];
  uint32_t sum = 0, nz = 0;
#pragma unroll
  for (int e = 0; e < kPer; ++e) {
    const int k = t * kPer + e;
    v[e] = k < tiles ? s->tile_sum[k] : 0u;
    sum += v[e];
    nz += k < tiles ? s->tile_nz[k] : 0u;
  }
  uint32_t total;
  uint32_t run = block_exclusive_scan(sum, scan, &total);
#pragma unroll
  for (int e = 0; e < kPer; ++e) {
    first[t * kPer + e] = run;
    run += v[e];
  }
  if (t == 0) first[tiles] = total;
  uint32_t dtot;
  block_exclusive_scan(nz, scan, &dtot);  // ends with a barrier: `first` is complete
  if (blockIdx.x == 0 && t == 0) *distinct = (int32_t)dtot;
  for (int p = blockIdx.x * kTileThreads + t; p < c; p += gridDim.x * kTileThreads) {
    int lo = 0, hi = tiles - 1;  // last tile with first[tile] <= p
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (first[mid] <= (uint32_t)p)
        lo = mid;
      else
        hi = mid - 1;
    }
    const uint32_t r = (uint32_t)p - first[lo];
    const int c0 = lo * kTile;
    const int cn = min(kTile, n - c0);
    const uint32_t* pre = s->count + c0;
    int a = 0, b = cn - 1;  // first column of the tile whose inclusive prefix exceeds r
    while (a < b) {
      const int mid = (a + b) >> 1;
      if (pre[mid] <= r)
        a = mid + 1;
      else
        b = mid;
    }
    out[p] = (uint32_t)(c0 + a);
  }
}

// Address of g_scratch on the current device (resolved on every call, so that a context torn
// down and recreated, which reloads the module, never leaves a stale address behind).
int scratch_for_current_device(NoAllocScratch** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
  if (e != cudaSuccess) return record_cuda_failure(e, "cudaGetSymbolAddress(g_scratch)");
  *out = static_cast<NoAllocScratch*>(p);
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
  int expand_blocks = (ci + kTileThreads - 1) / kTileThreads;
  if (expand_blocks > 1024) expand_blocks = 1024;
  expand_kernel<<<expand_blocks, kTileThreads, 0, st>>>(s, ni, tiles, ci, d_idx_sorted,
                                                        d_distinct);
  count_launch(4);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return record_cuda_failure(e, "amm_pick_sorted_noalloc launch");
  return AMM_OK;
}
