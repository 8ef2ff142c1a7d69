// CUDA kernels of libamm (sm_100a).
//
// A power-method call, all stream-ordered with no host round trip:
//   init_kernel      x0, the memo pair, the first state
//   sample_kernel,   every kListWindow steps: the picks (xorshift32 + inverse CDF) of the next
//   compact_kernel   kListWindow AMM steps and their sorted distinct work lists
//   panel_kernel     one launch per step (amm_panel.cu): the product over the step's columns,
//                    the grid-wide reduction into y and the Rayleigh quotient / next state
//   finalize_kernel  x_final, y_final, the committed sampling states
// plus the CDF construction of the set-up and the standalone helpers.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstdlib>
#include <utility>

#include "amm_device.cuh"
#include "amm_internal.h"

namespace amm {

static std::atomic<int64_t> g_launches{0};
void count_launch(int k) { g_launches.fetch_add(k, std::memory_order_relaxed); }
int64_t launch_count() { return g_launches.load(std::memory_order_relaxed); }

// The per-call kernels are launched as programmatic dependents of the kernel before them in the
// stream (each waits for it with griddep_wait before touching global memory), so that their
// launch overlaps the previous kernel's tail.  AMM_PDL=0 turns it off, for comparison.
bool pdl_enabled() {
  static const bool on = [] {
    const char* v = getenv("AMM_PDL");
    return !(v && *v && atoi(v) == 0);
  }();
  return on;
}

template <typename... P, typename... A>
static cudaError_t launch_pdl(void (*k)(P...), dim3 grid, dim3 block, cudaStream_t s,
                              A&&... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl_enabled() ? 1 : 0;
  const cudaError_t e = cudaLaunchKernelEx(&cfg, k, std::forward<A>(args)...);
  count_launch();
  return e != cudaSuccess ? e : cudaGetLastError();
}


// First index i in [0, n) with cdf[i] > target, else n-1 (device_memory.h:529-543).
// The coarse table (in shared memory) holds cdf[(s+1)*seg - 1] for the ncoarse full segments;
// the final window of kSeg elements is counted with independent vector loads.
template <typename F>
__device__ __forceinline__ uint32_t search_cdf(const F* __restrict__ cdf, const F* coarse,
                                               int ncoarse, int seg, int n, F target) {
  // number of full segments whose last value is <= target
  int lo = 0, hi = ncoarse;  // answer in [lo, hi]
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (coarse[mid] <= target)
      lo = mid + 1;
    else
      hi = mid;
  }
  int base, len;
  if (lo < ncoarse) {
    base = lo * seg;  // answer inside [base, base+seg); cdf[base+seg-1] > target
    len = seg;
    while (len > kSeg) {  // bisection in global memory down to one window
      const int half = len >> 1;
      if (cdf[base + half - 1] <= target) base += half;
      len = half;
    }
    // count values <= target in the window (monotone: = offset of the first value > target)
    int cnt = 0;
    constexpr int V = 16 / sizeof(F);
    const uint4* w = reinterpret_cast<const uint4*>(cdf + base);
#pragma unroll
    for (int k = 0; k < kSeg / V; ++k) {
      const uint4 q = __ldg(w + k);
      const F* f = reinterpret_cast<const F*>(&q);
#pragma unroll
      for (int e = 0; e < V; ++e) cnt += (f[e] <= target) ? 1 : 0;
    }
    return static_cast<uint32_t>(base + cnt);
  }
  // tail past the full segments
  base = ncoarse * seg;
  int cnt = 0;
  for (int k = base; k < n; ++k) cnt += (__ldg(cdf + k) <= target) ? 1 : 0;
  const int idx = base + cnt;
  return static_cast<uint32_t>(idx < n ? idx : n - 1);
}

// Draw the picks of AMM step number `list` of a call for samples k = k0, k0+kstride, ... < c:
// sample k uses its call-start state advanced list+1 times (one xorshift32 per AMM step, as the
// reference's one draw per state per step).  Writes the raw picks and the multiplicity histogram.
template <typename F>
__device__ void draw_samples(const Buffers& b, int which, const uint32_t* __restrict__ st_in,
                             int list, uint32_t* __restrict__ count, uint32_t* __restrict__ chunk,
                             uint32_t* __restrict__ samples, int k0, int kstride,
                             const F* coarse_s) {
  const F* cdf = nullptr;
  if constexpr (sizeof(F) == 8)
    cdf = reinterpret_cast<const F*>(b.cdf64[which]);
  else
    cdf = reinterpret_cast<const F*>(b.cdf32[which]);
  const F total = cdf[b.n - 1];
  for (int k = k0; k < b.c; k += kstride) {
    uint32_t y = st_in[k];
    for (int r = 0; r <= list; ++r) y = xorshift32(y);
    const float u = uniform_from(y);
    F target;
    if constexpr (sizeof(F) == 8)
      target = __dmul_rn(total, static_cast<double>(u));
    else
      target = __fmul_rn(total, u);
    const uint32_t idx = search_cdf<F>(cdf, coarse_s, b.ncoarse, b.seg, b.n, target);
    samples[k] = idx;
    const uint32_t old = atomicAdd(count + idx, 1u);
    if (old == 0u) atomicAdd(chunk + (idx >> b.chunk_shift), 1u);
  }
}

template <typename F>
__device__ void load_coarse(const Buffers& b, int which, F* coarse_s) {
  const F* src;
  if constexpr (sizeof(F) == 8)
    src = reinterpret_cast<const F*>(b.coarse64[which]);
  else
    src = reinterpret_cast<const F*>(b.coarse32[which]);
  // asynchronous 16-byte copies (every copy in flight at once; the table and its shared-memory
  // copy are 16-byte aligned), the odd tail by plain loads
  constexpr int V = 16 / (int)sizeof(F);
  const int nv = b.ncoarse / V;
  for (int k = threadIdx.x; k < nv; k += blockDim.x) cp_async16(coarse_s + k * V, src + k * V);
  for (int k = nv * V + threadIdx.x; k < b.ncoarse; k += blockDim.x) coarse_s[k] = __ldg(src + k);
  cp_async_wait_all();
  __syncthreads();
}

// ------------------------------------------------------------------------------------------
// Sampling (pick_index, device_memory.h:516-545), one sample per thread
// ------------------------------------------------------------------------------------------
struct SampleArgs {
  Buffers b;
  CallCfg cc;
  int iter;     // the window is refilled ahead of step `iter` (a multiple of kListWindow)
};

// List number st.drawn + blockIdx.y of the window ahead of step iter, drawn from the call-start
// states states[0] into its slot, if the window reaches it (see window_end).  The lists of the
// window are drawn by independent grid rows.
template <typename F>
__global__ void __launch_bounds__(256) sample_kernel(const __grid_constant__ SampleArgs a) {
  griddep_wait();
  griddep_launch_dependents();
  __shared__ __align__(16) F coarse_s[kCoarseMax];
  const Buffers& b = a.b;
  const CallCfg& cc = a.cc;
  const IterState& st = b.st[a.iter & 1];
  const int list = st.drawn + (int)blockIdx.y;
  if (st.done || list >= window_end(cc, a.iter, st)) return;  // uniform over the CTA
  const int slot = list % kListWindow;
  const int which = list_weighting(cc, list);
  load_coarse<F>(b, which, coarse_s);
  draw_samples<F>(b, which, b.states[0], list, b.count[slot], b.chunk[slot], b.samples[slot],
                  blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x, coarse_s);
}

// Sorted distinct work lists of the picks just drawn (the product kernel's column lists): per
// list (grid row) one CTA per kCompactSpan columns counts the picked columns below its range,
// scans its own range in column order and writes (column, w_j · multiplicity, α_j) at each picked
// column's rank; CTA 0 of the row also writes the list length.  It makes the same decision as
// sample_kernel and runs after it on the same stream.  The picks of the first list of a call are
// also kept as (index, multiplicity) for the single-product entry points.
constexpr int kCompactThreads = 256;
constexpr int kCompactPer = 4;
constexpr int kCompactSpan = kCompactThreads * kCompactPer;

__global__ void __launch_bounds__(kCompactThreads) compact_kernel(const __grid_constant__ SampleArgs a) {
  griddep_wait();
  griddep_launch_dependents();
  __shared__ uint32_t scan[40];
  const Buffers& b = a.b;
  const CallCfg& cc = a.cc;
  const IterState& st = b.st[a.iter & 1];
  const int list = st.drawn + (int)blockIdx.y;
  if (st.done || list >= window_end(cc, a.iter, st)) return;  // uniform over the CTA
  const int slot = list % kListWindow;
  const int which = list_weighting(cc, list);
  const uint32_t* __restrict__ cnt = b.count[slot];
  const uint32_t* __restrict__ chunk = b.chunk[slot];
  const int t = threadIdx.x;
  const int start = blockIdx.x * kCompactSpan;
  // picked columns below `start`: the whole chunks, then the columns of the chunk `start` is in
  const int c_lo = start >> b.chunk_shift;
  uint32_t below = 0;
  for (int k = t; k < c_lo; k += kCompactThreads) below += __ldg(chunk + k);
  for (int j = (c_lo << b.chunk_shift) + t; j < start; j += kCompactThreads)
    below += (__ldg(cnt + j) != 0u) ? 1u : 0u;
  uint32_t base;
  block_exclusive_scan(below, scan, &base);
  if (blockIdx.x == 0) {
    uint32_t all = 0;
    for (int k = t; k < b.nchunks; k += kCompactThreads) all += __ldg(chunk + k);
    uint32_t total;
    block_exclusive_scan(all, scan, &total);
    if (t == 0) b.wl_count[slot] = total;
  }
  uint32_t mult[kCompactPer];
  uint32_t nz = 0;
  const int j0 = start + t * kCompactPer;
#pragma unroll
  for (int e = 0; e < kCompactPer; ++e) {
    const int j = j0 + e;
    mult[e] = j < b.n ? __ldg(cnt + j) : 0u;
    nz += mult[e] ? 1u : 0u;
  }
  uint32_t unused;
  uint32_t r = base + block_exclusive_scan(nz, scan, &unused);
  const float* __restrict__ wts = b.wts[which];
  uint32_t* __restrict__ wl_col = b.wl_col[slot];
  float* __restrict__ wl_wm = b.wl_wm[slot];
  float* __restrict__ wl_al = b.wl_al[slot];
#pragma unroll
  for (int e = 0; e < kCompactPer; ++e) {
    if (mult[e]) {
      const int j = j0 + e;
      wl_col[r] = (uint32_t)j;
      wl_wm[r] = __fmul_rn(__ldg(wts + j), (float)mult[e]);
      wl_al[r] = __ldg(b.alpha + j);
      if (list == 0) {
        b.distinct_idx[r] = (uint32_t)j;
        b.distinct_mult[r] = mult[e];
      }
      ++r;
    }
  }
}

// A caller-supplied work list (amm_core_list_product): α_j of each listed column, and no index
// outside the matrix reaches the product kernel.
__global__ void __launch_bounds__(256) gather_alpha_kernel(const __grid_constant__ Buffers b,
                                                           int count) {
  griddep_wait();
  griddep_launch_dependents();
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
    uint32_t col = b.wl_col[0][k];
    if (col >= (uint32_t)b.n) {
      b.wl_col[0][k] = 0u;
      b.wl_wm[0][k] = 0.0f;
      col = 0u;
      atomicOr(b.status, (uint32_t)kDevBadIndex);
    }
    b.wl_al[0][k] = __ldg(b.alpha + col);
  }
}

// ------------------------------------------------------------------------------------------
// One rank's share of a draw over a column-sharded matrix (amm_shard_product): the c picks
// are drawn from the GLOBAL inclusive CDF (every rank draws the same picks from the same
// states), and the picks that fall in this rank's columns [col0, col0 + n) become its work list
// in slot 0, with w = multiplicity·total/(c·(cdf[j] − cdf[j−1])) (the realised probability of
// the draw) and the column's α.
// ------------------------------------------------------------------------------------------
struct ShardArgs {
  Buffers b;
  const double* cdf;   // global inclusive CDF, n_global entries
  int n_global;
  int col0;            // first global column of this rank
  const uint32_t* st_in;
  uint32_t* st_out;
  int c;
};

__global__ void __launch_bounds__(256) shard_draw_kernel(const __grid_constant__ ShardArgs a) {
  griddep_wait();
  griddep_launch_dependents();
  const double total = __ldg(a.cdf + a.n_global - 1);
  uint32_t* cnt = a.b.count[0];
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < a.c; k += gridDim.x * blockDim.x) {
    const uint32_t y = xorshift32(a.st_in[k]);  // get_rand (device_memory.h:506-514)
    a.st_out[k] = y;
    const double target = __dmul_rn(total, (double)uniform_from(y));
    int lo = 0, hi = a.n_global;  // first i with cdf[i] > target, else n - 1 (:529-543)
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (__ldg(a.cdf + mid) <= target)
        lo = mid + 1;
      else
        hi = mid;
    }
    const int j = (lo < a.n_global ? lo : a.n_global - 1) - a.col0;
    if (j >= 0 && j < a.b.n) atomicAdd(cnt + j, 1u);
  }
}

constexpr int kShardThreads = 1024;

// One block: the picked local columns in ascending order (a block scan of the per-thread
// counts of non-zero multiplicities over contiguous column runs), their weights and α; the
// multiplicities are cleared for the next draw.
__global__ void __launch_bounds__(kShardThreads) shard_compact_kernel(
    const __grid_constant__ ShardArgs a) {
  griddep_wait();
  griddep_launch_dependents();
  __shared__ uint32_t scan[40];
  const Buffers& b = a.b;
  const int t = threadIdx.x;
  const int per = (b.n + kShardThreads - 1) / kShardThreads;
  const int j0 = t * per, j1 = min(b.n, j0 + per);
  uint32_t* cnt = b.count[0];
  uint32_t nz = 0;
  for (int j = j0; j < j1; ++j) nz += cnt[j] ? 1u : 0u;
  uint32_t total_nz;
  uint32_t r = block_exclusive_scan(nz, scan, &total_nz);
  const double total = __ldg(a.cdf + a.n_global - 1);
  for (int j = j0; j < j1; ++j) {
    const uint32_t mult = cnt[j];
    if (!mult) continue;
    const int jg = j + a.col0;
    const double step = __ldg(a.cdf + jg) - (jg > 0 ? __ldg(a.cdf + jg - 1) : 0.0);
    b.wl_col[0][r] = (uint32_t)j;
    b.wl_wm[0][r] = (float)((double)mult * total / ((double)a.c * step));
    b.wl_al[0][r] = __ldg(b.alpha + j);
    cnt[j] = 0u;
    ++r;
  }
  if (t == 0) b.wl_count[0] = total_nz;
}

// ------------------------------------------------------------------------------------------
// Call start / end
// ------------------------------------------------------------------------------------------
struct InitArgs {
  Buffers b;
  CallCfg cc;
  const float* x0;
  int no_normalize;
};

__global__ void __launch_bounds__(1024) init_kernel(const __grid_constant__ InitArgs a) {
  griddep_wait();
  griddep_launch_dependents();
  const Buffers& b = a.b;
  const CallCfg& cc = a.cc;
  const int t = threadIdx.x;
  __shared__ double ws[32];
  const float* __restrict__ x0 = a.x0;
  float* __restrict__ y1 = b.y[1];
  double ss = 0.0;
  // a call starts from a zero memo pair, as the reference's zero_clear (device_memory.h:
  // 345-355, called first by every powerMethod_by_*); the single-product entry points keep
  // the memo their caller supplied
  const bool clear_memo = !a.no_normalize;
#pragma unroll 4
  for (int k0 = 4 * t; k0 < b.m; k0 += 4 * blockDim.x) {  // m % 4 == 0
    const float4 v = __ldg(reinterpret_cast<const float4*>(x0 + k0));
    *reinterpret_cast<float4*>(y1 + k0) = v;
    if (clear_memo) {
      *reinterpret_cast<float4*>(b.x_memo + k0) = make_float4(0.f, 0.f, 0.f, 0.f);
      *reinterpret_cast<float4*>(b.y_memo + k0) = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    ss = fma((double)v.x, (double)v.x, ss);
    ss = fma((double)v.y, (double)v.y, ss);
    ss = fma((double)v.z, (double)v.z, ss);
    ss = fma((double)v.w, (double)v.w, ss);
  }
  ss = warp_sum(ss);
  if ((t & 31) == 0) ws[t >> 5] = ss;
  __syncthreads();
  if (t == 0) {
    b.ticket[2] = 0u;  // the step kernels' grid-barrier count
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += ws[w];
    IterState st{};
    st.scale = a.no_normalize ? 1.0f : (float)rsqrt(s);  // normalize (common.h:156-183)
    st.cos_prev = 0.0;
    st.lam_prev = 0.0;
    int le;
    st.mode = decide_mode(cc, 0, 0.0, 0, &le);
    st.last_exact = le;
    st.done = 0;
    st.used = 0;
    st.drawn = 0;
    st.steps_run = 0;
    st.memo_zero = clear_memo ? 1 : 0;
    if (!(s > 0.0) || !isfinite(s)) {
      atomicOr(b.status, (uint32_t)kDevNonFinite);
      st.done = 1;
    }
    b.st[0] = st;
    b.tstamp[0] = globaltimer_ns();
  }
}

constexpr int kFinalThreads = 256;

struct FinalArgs {
  Buffers b;
  CallCfg cc;
  float* xdst;
  float* ydst;
};

__global__ void __launch_bounds__(kFinalThreads) finalize_kernel(const __grid_constant__ FinalArgs a) {
  griddep_wait();
  griddep_launch_dependents();
  const Buffers& b = a.b;
  const IterState st = b.st[a.cc.step & 1];
  const int gt = blockIdx.x * blockDim.x + threadIdx.x, gs = gridDim.x * blockDim.x;
  const int last = st.steps_run - 1;
  const float* ylast = last >= 0 ? b.y[last & 1] : b.y[1];
  for (int k = gt; k < b.m; k += gs) {
    const float yv = ylast[k];
    if (a.xdst) a.xdst[k] = __fmul_rn(st.scale, yv);
    if (a.ydst) a.ydst[k] = yv;
  }
  if (a.cc.uses_amm && !a.cc.sanity && !a.cc.ext_list) {
    // commit: each state advanced once per AMM step that ran
    if (st.used > 0)
      for (int k = gt; k < b.c; k += gs) {
        uint32_t y = b.states[0][k];
        for (int r = 0; r < st.used; ++r) y = xorshift32(y);
        b.states[0][k] = y;
      }
    // pending (drawn ahead, never consumed) lists are dropped: their states are not committed
    for (int list = st.used; list < st.drawn; ++list) {
      const int slot = list % kListWindow;
      uint32_t* cnt = b.count[slot];
      const uint32_t* smp = b.samples[slot];
      for (int k = gt; k < b.c; k += gs) cnt[smp[k]] = 0u;
      for (int k = gt; k < b.nchunks; k += gs) b.chunk[slot][k] = 0u;
    }
  }
}

// ------------------------------------------------------------------------------------------
// CDF construction (once per matrix): tile sums, then tile scans with the ordered prefix of the
// preceding tiles (deterministic association).  FP64 mode: weight_j = (double)norm_j²; FP32
// mode: weight_j = fl32(norm_j²) as set_weights (common.h:34-40) and the CDF is fl32 of the
// FP64 prefix.  Then w_j = total/(weight_j·c) (update_weights, common.h:42-53) and the coarse
// table of the sampler.
// ------------------------------------------------------------------------------------------
constexpr int kCdfThreads = 256;
constexpr int kCdfPer = kCdfTile / kCdfThreads;  // kCdfTile: amm_internal.h


// Block-wide exclusive scan of one double per thread (kCdfThreads threads); total in *total.
__device__ double block_exclusive_scan_f64(double v, double* ws, double* total) {
  // ws: >= 33 doubles
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int nw = kCdfThreads / 32;
  double incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const double y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) ws[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    const double w = lane < nw ? ws[lane] : 0.0;
    double wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const double y = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += y;
    }
    if (lane < nw) ws[lane] = wi - w;
    if (lane == nw - 1) ws[32] = wi;
  }
  __syncthreads();
  const double r = ws[warp] + (incl - v);
  *total = ws[32];
  __syncthreads();
  return r;
}

// Local (within-tile) inclusive prefix of this thread's kCdfPer weights and the tile total,
// computed identically by both CDF kernels: a thread-sequential sum, a block scan of the thread
// sums, then thread-sequential accumulation.  The tile total is the last local prefix value,
// so cdf = pre_tile + local_prefix is non-decreasing across tile boundaries as well.
__device__ void tile_local_prefix(const Buffers& b, const float* base, int t0, int sanity,
                                  double (&lp)[kCdfPer], double* tile_total, double* ws,
                                  float* tile) {
  const float* __restrict__ src = base;
#pragma unroll 4
  for (int k = threadIdx.x; k < kCdfTile; k += kCdfThreads) {
    const int j = t0 + k;
    tile[k] = j < b.n ? __ldg(src + j) : 0.f;
  }
  __syncthreads();
  double w[kCdfPer];
  double loc = 0.0;
#pragma unroll
  for (int e = 0; e < kCdfPer; ++e) {
    const int k = threadIdx.x * kCdfPer + e;
    const float nv = tile[k];
    w[e] = (t0 + k < b.n)
               ? (sanity ? 1.0 : (b.cdf_f32 ? (double)__fmul_rn(nv, nv) : (double)nv * (double)nv))
               : 0.0;
    loc += w[e];
  }
  double unused;
  double run = block_exclusive_scan_f64(loc, ws, &unused);
#pragma unroll
  for (int e = 0; e < kCdfPer; ++e) {
    run += w[e];
    lp[e] = run;
  }
  if (threadIdx.x == kCdfThreads - 1) ws[33] = run;
  __syncthreads();
  *tile_total = ws[33];
  __syncthreads();
}

// grid (ntiles, weightings): the total of each tile
__global__ void __launch_bounds__(kCdfThreads) cdf_tile_sums_kernel(const __grid_constant__ Buffers b,
                                                                   int which0, int sanity) {
  griddep_wait();
  griddep_launch_dependents();
  __shared__ double ws[34];
  __shared__ float tile[kCdfTile];
  const int which = which0 + blockIdx.y;
  const float* base = which == 0 ? b.norm : b.normp;
  double lp[kCdfPer], tot;
  tile_local_prefix(b, base, blockIdx.x * kCdfTile, sanity, lp, &tot, ws, tile);
  if (threadIdx.x == 0) b.cdf_tsum[which * gridDim.x + blockIdx.x] = tot;
}

// grid (ntiles, weightings): CDF of each tile (unless imported), weights w_j
__global__ void __launch_bounds__(kCdfThreads) cdf_scan_kernel(const __grid_constant__ Buffers b,
                                                               int which0, int keep_cdf, int sanity) {
  griddep_wait();
  griddep_launch_dependents();
  __shared__ double ws[34];
  __shared__ float tile[kCdfTile];
  __shared__ double pre_s, total_s;
  const int which = which0 + blockIdx.y;
  const float* base = which == 0 ? b.norm : b.normp;
  const int ntiles = gridDim.x;
  const int t0 = blockIdx.x * kCdfTile;
  const int n = b.n;
  double total64;
  if (!keep_cdf) {
    // prefixes and the total summed sequentially in tile order (identical in every block);
    // the tile sums are first staged in shared memory by all threads
    double* ts = reinterpret_cast<double*>(tile);  // reused before the tile is loaded
    const int nts = ntiles < kCdfTile / 2 ? ntiles : kCdfTile / 2;
    for (int k = threadIdx.x; k < nts; k += kCdfThreads) ts[k] = __ldcg(b.cdf_tsum + which * ntiles + k);
    __syncthreads();
    if (threadIdx.x == 0) {
      double acc = 0.0, pre = 0.0;
      for (int k = 0; k < ntiles; ++k) {
        if (k == (int)blockIdx.x) pre = acc;
        acc += k < nts ? ts[k] : __ldcg(b.cdf_tsum + which * ntiles + k);
      }
      pre_s = pre;
      total_s = acc;
    }
    __syncthreads();
    double lp[kCdfPer], tot;
    tile_local_prefix(b, base, t0, sanity, lp, &tot, ws, tile);
    const double pre = pre_s;
#pragma unroll
    for (int e = 0; e < kCdfPer; ++e) {
      const int j = t0 + threadIdx.x * kCdfPer + e;
      if (j < n) {
        const bool seg_end = ((j + 1) & (b.seg - 1)) == 0 && (j + 1) / b.seg <= b.ncoarse;
        if (b.cdf_f32) {
          const float cv = (float)(pre + lp[e]);
          b.cdf32[which][j] = cv;
          if (seg_end) b.coarse32[which][(j + 1) / b.seg - 1] = cv;
        } else {
          const double cv = pre + lp[e];
          b.cdf64[which][j] = cv;
          if (seg_end) b.coarse64[which][(j + 1) / b.seg - 1] = cv;
        }
      }
    }
    total64 = total_s;
  } else {
    total64 = b.cdf_f32 ? (double)b.cdf32[which][n - 1] : b.cdf64[which][n - 1];
    // the coarse table of the imported CDF: the last value of each full segment
    for (int k = threadIdx.x; k < kCdfTile; k += kCdfThreads) {
      const int j = t0 + k;
      if (j < n && ((j + 1) & (b.seg - 1)) == 0 && (j + 1) / b.seg <= b.ncoarse) {
        if (b.cdf_f32)
          b.coarse32[which][(j + 1) / b.seg - 1] = b.cdf32[which][j];
        else
          b.coarse64[which][(j + 1) / b.seg - 1] = b.cdf64[which][j];
      }
    }
  }
  const float total32 = b.cdf_f32 ? (float)total64 : 0.f;
  for (int k = threadIdx.x; k < kCdfTile; k += kCdfThreads) {
    const int j = t0 + k;
    if (j >= n) break;
    const float nv = base[j];
    float w;
    if (b.cdf_f32) {
      const float w32 = sanity ? 1.0f : __fmul_rn(nv, nv);
      w = __fdiv_rn(total32, __fmul_rn(w32, (float)b.c));
    } else {
      const double w64 = sanity ? 1.0 : (double)nv * (double)nv;
      w = (float)(total64 / (w64 * (double)b.c));
    }
    b.wts[which][j] = w;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && (!(total64 > 0.0) || !isfinite(total64)))
    atomicOr(b.status, (uint32_t)kDevNonFinite);
}

__global__ void __launch_bounds__(512) normalize_kernel(float* x, int m) {
  __shared__ double ws[16];
  __shared__ float scale_s;
  const int t = threadIdx.x;
  double ss = 0.0;
  for (int k = t; k < m; k += blockDim.x) ss = fma((double)x[k], (double)x[k], ss);
  ss = warp_sum(ss);
  if ((t & 31) == 0) ws[t >> 5] = ss;
  __syncthreads();
  if (t == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += ws[w];
    scale_s = (float)rsqrt(s);
  }
  __syncthreads();
  for (int k = t; k < m; k += blockDim.x) x[k] = __fmul_rn(x[k], scale_s);
}

__global__ void __launch_bounds__(512) rayleigh_kernel(const float* x_in, float* x_out,
                                                       const float* y, const double* vstar, int m,
                                                       double* out3) {
  __shared__ double ws[16][3];
  __shared__ float scale_s;
  const int t = threadIdx.x;
  double xy = 0.0, yy = 0.0, yv = 0.0;
  for (int k = t; k < m; k += blockDim.x) {
    const double yd = (double)y[k];
    xy = fma(yd, (double)x_in[k], xy);
    yy = fma(yd, yd, yy);
    if (vstar) yv = fma(yd, vstar[k], yv);
  }
  xy = warp_sum(xy);
  yy = warp_sum(yy);
  yv = warp_sum(yv);
  if ((t & 31) == 0) {
    ws[t >> 5][0] = xy;
    ws[t >> 5][1] = yy;
    ws[t >> 5][2] = yv;
  }
  __syncthreads();
  if (t == 0) {
    double a = 0, c = 0, e = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      a += ws[w][0];
      c += ws[w][1];
      e += ws[w][2];
    }
    const double sc = rsqrt(c);
    out3[0] = a;
    out3[1] = e * sc;
    out3[2] = a * sc;
    scale_s = (float)sc;
  }
  __syncthreads();
  for (int k = t; k < m; k += blockDim.x) x_out[k] = __fmul_rn(scale_s, y[k]);
}

// Draw c indices from states[0] without storing the advanced states.
template <typename F>
__global__ void __launch_bounds__(256) sample_only_kernel(const __grid_constant__ Buffers b,
                                                          int which, uint32_t* idx) {
  __shared__ __align__(16) F coarse_s[kCoarseMax];
  load_coarse<F>(b, which, coarse_s);
  const F* cdf;
  if constexpr (sizeof(F) == 8)
    cdf = reinterpret_cast<const F*>(b.cdf64[which]);
  else
    cdf = reinterpret_cast<const F*>(b.cdf32[which]);
  const F total = cdf[b.n - 1];
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < b.c; k += gridDim.x * blockDim.x) {
    const float u = uniform_from(xorshift32(b.states[0][k]));
    F target;
    if constexpr (sizeof(F) == 8)
      target = __dmul_rn(total, static_cast<double>(u));
    else
      target = __fmul_rn(total, u);
    idx[k] = search_cdf<F>(cdf, coarse_s, b.ncoarse, b.seg, b.n, target);
  }
}

// Expand the sorted distinct list (index, multiplicity) of the last AMM product into the
// sorted index multiset of length c (single CTA).
__global__ void __launch_bounds__(1024) expand_sorted_kernel(const __grid_constant__ Buffers b,
                                                             const int32_t* d_cd, uint32_t* out) {
  __shared__ uint32_t scan[40];
  const int cd = *d_cd;
  uint32_t carry = 0;
  for (int base = 0; base < cd; base += blockDim.x) {
    const int k = base + threadIdx.x;
    const uint32_t mult = k < cd ? b.distinct_mult[k] : 0u;
    uint32_t tot;
    const uint32_t ex = block_exclusive_scan(mult, scan, &tot);
    if (k < cd)
      for (uint32_t r = 0; r < mult; ++r)
        if (carry + ex + r < (uint32_t)b.c) out[carry + ex + r] = b.distinct_idx[k];
    carry += tot;
  }
}

// ∂λ/∂A = 2·v·(vᵀA): u_j = A_jᵀ v per column (warp per column), then the outer product.
template <typename Elem>
__global__ void __launch_bounds__(256) grad_colvec_kernel(const __grid_constant__ Buffers b,
                                                          const float* v, float* u) {
  const int lane = threadIdx.x & 31;
  const int wglob = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  const Elem* A = reinterpret_cast<const Elem*>(b.A);
  for (int j = wglob; j < b.n; j += nw) {
    const Elem* col = A + (size_t)j * b.ld;
    double s = 0.0;
    for (int r = lane; r < b.m; r += 32) {
      float a;
      if constexpr (sizeof(Elem) == 4)
        a = col[r];
      else
        a = __bfloat162float(col[r]);
      s = fma((double)a, (double)v[r], s);
    }
    s = warp_sum(s);
    if (lane == 0) u[j] = (float)s;
  }
}

// grid.x = columns, grid.y = row blocks of blockDim.x rows
__global__ void __launch_bounds__(256) grad_outer_kernel(const float* v, const float* u, int m,
                                                         int n, float* grad, int64_t ldg) {
  const int j = blockIdx.x;
  const int r = blockIdx.y * blockDim.x + threadIdx.x;
  if (j < n && r < m) grad[(size_t)j * ldg + r] = 2.0f * v[r] * u[j];
}

// ------------------------------------------------------------------------------------------
// Host launchers
// ------------------------------------------------------------------------------------------
cudaError_t launch_build_cdf(const Buffers& b, int which, int keep_cdf, int sanity,
                             cudaStream_t s) {
  const int ntiles = (b.n + kCdfTile - 1) / kCdfTile;
  const dim3 grid(ntiles, which >= 0 ? 1 : 2);
  const int w0 = which >= 0 ? which : 0;
  if (!keep_cdf) {
    const cudaError_t e = launch_pdl(cdf_tile_sums_kernel, grid, dim3(kCdfThreads), s, b, w0, sanity);
    if (e != cudaSuccess) return e;
  }
  return launch_pdl(cdf_scan_kernel, grid, dim3(kCdfThreads), s, b, w0, keep_cdf, sanity);
}

cudaError_t launch_shard_worklist(const Buffers& b, const double* cdf, int n_global, int col0,
                                  const uint32_t* st_in, uint32_t* st_out, int c, cudaStream_t s) {
  ShardArgs a{};
  a.b = b;
  a.cdf = cdf;
  a.n_global = n_global;
  a.col0 = col0;
  a.st_in = st_in;
  a.st_out = st_out;
  a.c = c;
  int blocks = (c + 255) / 256;
  if (blocks > 1024) blocks = 1024;
  cudaError_t e = launch_pdl(shard_draw_kernel, dim3(blocks), dim3(256), s, a);
  if (e != cudaSuccess) return e;
  return launch_pdl(shard_compact_kernel, dim3(1), dim3(kShardThreads), s, a);
}

cudaError_t launch_gather_alpha(const Buffers& b, int64_t count, cudaStream_t s) {
  int blocks = (int)((count + 255) / 256);
  if (blocks > 1024) blocks = 1024;
  if (blocks < 1) blocks = 1;
  return launch_pdl(gather_alpha_kernel, dim3(blocks), dim3(256), s, b, (int)count);
}

cudaError_t launch_init(const Buffers& b, const CallCfg& cc, const float* x0, int no_normalize,
                        cudaStream_t s) {
  InitArgs a{};
  a.b = b;
  a.cc = cc;
  a.x0 = x0;
  a.no_normalize = no_normalize;
  return launch_pdl(init_kernel, dim3(1), dim3(1024), s, a);
}

cudaError_t launch_sample(const Buffers& b, const CallCfg& cc, int iter, cudaStream_t s) {
  SampleArgs a{};
  a.b = b;
  a.cc = cc;
  a.iter = iter;
  int blocks = (b.c + 255) / 256;
  if (blocks > 1024) blocks = 1024;
  const int rows = cc.step < kListWindow ? cc.step : kListWindow;
  if (b.cdf_f32) return launch_pdl(sample_kernel<float>, dim3(blocks, rows), dim3(256), s, a);
  return launch_pdl(sample_kernel<double>, dim3(blocks, rows), dim3(256), s, a);
}

cudaError_t launch_compact(const Buffers& b, const CallCfg& cc, int iter, cudaStream_t s) {
  SampleArgs a{};
  a.b = b;
  a.cc = cc;
  a.iter = iter;
  const int blocks = (b.n + kCompactSpan - 1) / kCompactSpan;
  const int rows = cc.step < kListWindow ? cc.step : kListWindow;
  return launch_pdl(compact_kernel, dim3(blocks, rows), dim3(kCompactThreads), s, a);
}

cudaError_t launch_finalize(const Buffers& b, const CallCfg& cc, float* xdst, float* ydst,
                            cudaStream_t s) {
  FinalArgs a{};
  a.b = b;
  a.cc = cc;
  a.xdst = xdst;
  a.ydst = ydst;
  int blocks = (b.m + kFinalThreads - 1) / kFinalThreads;
  if (blocks > 256) blocks = 256;
  return launch_pdl(finalize_kernel, dim3(blocks), dim3(kFinalThreads), s, a);
}

__global__ void clock_kernel(unsigned long long* out) { *out = globaltimer_ns(); }

// The failure path of the library's bounded waits, run on purpose: one CTA waits on an mbarrier
// that nothing arrives on, then on a grid barrier that counts one CTA more than the grid.  Each
// wait gives up after kWaitLimitNs and the kernel records kDevTimeout in the status word, as the
// step kernels do; out[0..1]: whether each wait completed (0: gave up), out[2]: µs spent.
__global__ void wait_probe_kernel(uint32_t* status, uint32_t* counter, uint32_t* out) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_barrier_init();
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  const unsigned long long t0 = globaltimer_now();
  const bool a = mbar_wait_bounded(&bar, 0u);
  const bool g = grid_barrier(counter, gridDim.x + 1u);
  out[0] = a ? 1u : 0u;
  out[1] = g ? 1u : 0u;
  out[2] = (uint32_t)((globaltimer_now() - t0) / 1000ull);
  if (!a || !g) atomicOr(status, (uint32_t)kDevTimeout);
}

cudaError_t launch_wait_probe(uint32_t* status, uint32_t* counter, uint32_t* out,
                              cudaStream_t s) {
  wait_probe_kernel<<<1, 32, 0, s>>>(status, counter, out);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_clock(unsigned long long* out, cudaStream_t s) {
  clock_kernel<<<1, 1, 0, s>>>(out);
  count_launch();
  return cudaGetLastError();
}

// n floats (n % 4 == 0, both 16-byte aligned), as a programmatic dependent of the kernel before
// it: a device copy that does not leave the chain of kernel launches
__global__ void __launch_bounds__(256) copy4_kernel(float4* __restrict__ dst,
                                                    const float4* __restrict__ src, int n4) {
  griddep_wait();
  griddep_launch_dependents();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += gridDim.x * blockDim.x)
    dst[i] = src[i];
}

cudaError_t launch_copy(float* dst, const float* src, int n, cudaStream_t s) {
  if ((n & 3) || ((reinterpret_cast<uintptr_t>(dst) | reinterpret_cast<uintptr_t>(src)) & 15))
    return cudaMemcpyAsync(dst, src, sizeof(float) * n, cudaMemcpyDeviceToDevice, s);
  const int n4 = n / 4;
  int blocks = (n4 + 255) / 256;
  if (blocks > 64) blocks = 64;
  return launch_pdl(copy4_kernel, dim3(blocks), dim3(256), s, reinterpret_cast<float4*>(dst),
                    reinterpret_cast<const float4*>(src), n4);
}

cudaError_t launch_normalize(float* x, int m, cudaStream_t s) {
  normalize_kernel<<<1, 512, 0, s>>>(x, m);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_rayleigh(const float* x_in, float* x_out, const float* y, const double* vstar,
                            int m, double* out3, cudaStream_t s) {
  rayleigh_kernel<<<1, 512, 0, s>>>(x_in, x_out, y, vstar, m, out3);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_sample_only(const Buffers& b, int which, uint32_t* idx, cudaStream_t s) {
  const int blocks = (b.c + 255) / 256;
  if (b.cdf_f32)
    sample_only_kernel<float><<<blocks, 256, 0, s>>>(b, which, idx);
  else
    sample_only_kernel<double><<<blocks, 256, 0, s>>>(b, which, idx);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_expand_sorted(const Buffers& b, const int32_t* d_cd, uint32_t* out,
                                 cudaStream_t s) {
  expand_sorted_kernel<<<1, 1024, 0, s>>>(b, d_cd, out);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_grad(const Buffers& b, const float* v, float* grad, int64_t ldg,
                        cudaStream_t s) {
  float* u = b.colvec;
  if (b.dtype == 1)
    grad_colvec_kernel<__nv_bfloat16><<<(b.n + 7) / 8, 256, 0, s>>>(b, v, u);
  else
    grad_colvec_kernel<float><<<(b.n + 7) / 8, 256, 0, s>>>(b, v, u);
  dim3 grid(b.n, (b.m + 255) / 256);
  grad_outer_kernel<<<grid, 256, 0, s>>>(v, u, b.m, b.n, grad, ldg);
  count_launch(2);
  return cudaGetLastError();
}

}  // namespace amm
