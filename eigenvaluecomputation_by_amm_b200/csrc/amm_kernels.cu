// CUDA kernels of libamm (sm_100a).
//
// Hot path per power-method iteration i (all stream-ordered, no host round trip):
//   panel_kernel   one pass over the columns of this step (all n for an exact step, the
//                  distinct sampled columns for an AMM step): each column is brought into
//                  shared memory by a 1-D TMA bulk copy, dotted with dx, and the scaled
//                  column is accumulated into a per-CTA y in registers.  Each column is read
//                  from HBM once (the reference reads it twice: previousAMM_kernel1 and _2).
//   reduce_kernel  deterministic sum of the per-CTA partials, the rank-one terms of the
//                  proposed method, the memo copy of a VR step, the FP64 Rayleigh sums and
//                  (last CTA) λ, err, cos, the next scale and the next step's kind; extra
//                  CTAs draw the next step's samples (xorshift32 + inverse CDF) meanwhile.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>

#include "amm_internal.h"

namespace amm {

static std::atomic<int64_t> g_launches{0};
void count_launch(int k) { g_launches.fetch_add(k, std::memory_order_relaxed); }
int64_t launch_count() { return g_launches.load(std::memory_order_relaxed); }

// ------------------------------------------------------------------------------------------
// Device helpers
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait: gives up after ~2^22 polls (each try_wait may suspend briefly) and reports.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  for (uint32_t it = 0; it < (1u << 22); ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

__device__ __forceinline__ uint64_t l2_evict_first_policy() {
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}

// 1-D bulk copy global -> shared, completion signalled on `bar` (transaction bytes).
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar,
                                         uint64_t policy) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint "
      "[%0], [%1], %2, [%3], %4;" ::"r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar)), "l"(policy)
      : "memory");
}

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// 16-byte vector -> E floats.
__device__ __forceinline__ void unpack(const uint4& v, float (&o)[4]) {
  o[0] = __uint_as_float(v.x);
  o[1] = __uint_as_float(v.y);
  o[2] = __uint_as_float(v.z);
  o[3] = __uint_as_float(v.w);
}
__device__ __forceinline__ void unpack(const uint4& v, float (&o)[8]) {
  // bf16 -> fp32 is exact: the 16 bits become the high half of the float.
  o[0] = __uint_as_float(v.x << 16);
  o[1] = __uint_as_float(v.x & 0xffff0000u);
  o[2] = __uint_as_float(v.y << 16);
  o[3] = __uint_as_float(v.y & 0xffff0000u);
  o[4] = __uint_as_float(v.z << 16);
  o[5] = __uint_as_float(v.z & 0xffff0000u);
  o[6] = __uint_as_float(v.w << 16);
  o[7] = __uint_as_float(v.w & 0xffff0000u);
}

// Kind of the step that follows, as the reference's drivers decide it:
//  previous    powerMethod_by_previous.cuh:135-137
//  proposed    powerMethod_by_proposed.cuh:371-373 (no VR right after a VR step)
//  proposed_v2 powerMethod_by_proposed_v2.cuh:234-305
__device__ int decide_mode(const CallCfg& cc, int i, double cos_prev, int last_exact,
                           int* le_out) {
  *le_out = last_exact;
  const bool periodic = cc.vr_period > 0 && (i + 1) % cc.vr_period == 0;
  const bool adaptive = cc.vr_thr > 0.0 && cos_prev > 1.0 - cc.vr_thr;
  switch (cc.method) {
    case kMethodPrevious:
      return (cc.variance_reduction && (periodic || adaptive)) ? kExactMemo : kPrevious;
    case kMethodProposed:
      if (i > last_exact + 1 && cc.variance_reduction && (periodic || adaptive)) {
        *le_out = i;
        return kExactMemo;
      }
      return kProposed;
    case kMethodProposedV2:
      if (i < cc.vr_period - 1) return kPrevious;
      if (i == cc.vr_period - 1) return kExact;
      return (cc.variance_reduction && periodic) ? kExactMemo : kProposed;
    default:
      return kExact;
  }
}

// Weighting (0 = ‖A_j‖², 1 = ‖A_j − α_j‖²) of the first AMM step after step i.
__device__ __forceinline__ int next_amm_weighting(const CallCfg& cc, int i) {
  if (cc.method == kMethodPrevious) return 0;
  if (cc.method == kMethodProposed) return 1;
  if (cc.method == kMethodProposedV2) return (i + 1 < cc.vr_period - 1) ? 0 : 1;
  return 0;
}

__device__ __forceinline__ uint32_t xorshift32(uint32_t y) {
  y ^= (y << 13);
  y ^= (y >> 17);
  y ^= (y << 5);
  return y;
}
__device__ __forceinline__ float uniform_from(uint32_t y) {
  // exact: 1.mantissa - 1 (device_memory.h:513)
  return __fsub_rn(__uint_as_float((y & 0x007FFFFFu) | 0x3f800000u), 1.0f);
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

// Draw the picks of one AMM step for samples k = k0, k0+kstride, ... < c.
// Writes the advanced states, the raw picks and the multiplicity histogram.
template <typename F>
__device__ void draw_samples(const Buffers& b, int which, const uint32_t* __restrict__ st_in,
                             uint32_t* __restrict__ st_out, uint32_t* __restrict__ count,
                             uint32_t* __restrict__ chunk, uint32_t* __restrict__ samples, int k0,
                             int kstride, const F* coarse_s) {
  const F* cdf = nullptr;
  if constexpr (sizeof(F) == 8)
    cdf = reinterpret_cast<const F*>(b.cdf64[which]);
  else
    cdf = reinterpret_cast<const F*>(b.cdf32[which]);
  const F total = cdf[b.n - 1];
  for (int k = k0; k < b.c; k += kstride) {
    const uint32_t y = xorshift32(st_in[k]);
    st_out[k] = y;
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
  for (int k = threadIdx.x; k < b.ncoarse; k += blockDim.x) coarse_s[k] = src[k];
  __syncthreads();
}

// Sampling role shared by the init and reduce kernels: clear the consumed picks (optional)
// and draw the next ones.
__device__ void sampling_role(const Buffers& b, int which, int clear_pb, int sb_in, int pb_out,
                              int rank, int nranks, bool draw) {
  __shared__ __align__(16) double coarse_s[kCoarseMax];
  const int tid = rank * blockDim.x + threadIdx.x;
  const int nthr = nranks * blockDim.x;
  if (clear_pb >= 0) {
    uint32_t* cnt = b.count[clear_pb];
    const uint32_t* smp = b.samples[clear_pb];
    for (int k = tid; k < b.c; k += nthr) cnt[smp[k]] = 0u;
    for (int k = tid; k < b.nchunks; k += nthr) b.chunk[clear_pb][k] = 0u;
  }
  if (!draw) return;
  if (b.cdf_f32) {
    float* cs = reinterpret_cast<float*>(coarse_s);
    load_coarse<float>(b, which, cs);
    draw_samples<float>(b, which, b.states[sb_in], b.states[sb_in ^ 1], b.count[pb_out],
                        b.chunk[pb_out], b.samples[pb_out], tid, nthr, cs);
  } else {
    load_coarse<double>(b, which, coarse_s);
    draw_samples<double>(b, which, b.states[sb_in], b.states[sb_in ^ 1], b.count[pb_out],
                         b.chunk[pb_out], b.samples[pb_out], tid, nthr, coarse_s);
  }
}

// Block-wide exclusive scan of one uint32 per thread; returns the exclusive prefix and
// writes the block total to *total.  `scratch` holds >= 33 uint32.
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* scratch,
                                                         uint32_t* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  uint32_t incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) scratch[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < nw ? scratch[lane] : 0u;
    uint32_t wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += y;
    }
    if (lane < nw) scratch[lane] = wi - w;
    if (lane == 31) scratch[32] = wi;
  }
  __syncthreads();
  const uint32_t r = scratch[warp] + incl - v;
  *total = scratch[32];
  __syncthreads();
  return r;
}

// ------------------------------------------------------------------------------------------
// Panel kernel
// ------------------------------------------------------------------------------------------
struct PanelArgs {
  Buffers b;
  PanelGeom g;
  CallCfg cc;
  int iter;
  int setup;
};

// Shared memory: [stage_area >= nstages * stage_bytes] | bars[8] | red (4 KB) | wl_idx | wl_mult | scan[40]
template <typename Elem, int R, bool SETUP>
__global__ void __launch_bounds__(kMaxThreads, 1) panel_kernel(const __grid_constant__ PanelArgs a) {
  constexpr int E = 16 / static_cast<int>(sizeof(Elem));
  const Buffers& b = a.b;
  const PanelGeom& g = a.g;
  const int T = blockDim.x, t = threadIdx.x, warp = t >> 5, lane = t & 31, nwarps = T >> 5;
  const int m = b.m, nvec = m / E, G = gridDim.x, bid = blockIdx.x;

  extern __shared__ __align__(128) unsigned char smem[];
  unsigned char* stage_base = smem;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + (size_t)g.stage_area);
  float* red = reinterpret_cast<float*>(bars + 8);
  double* red64 = reinterpret_cast<double*>(red);
  uint32_t* wl_idx = reinterpret_cast<uint32_t*>(reinterpret_cast<unsigned char*>(red) + 4096);
  uint32_t* wl_mult = wl_idx + g.wl_cap;
  uint32_t* scan = wl_mult + g.wl_cap;

  int mode = kExact, pb = 0;
  float scale = 0.f;
  if (!SETUP) {
    const IterState& st = b.st[a.iter & 1];
    if (st.done) return;
    mode = st.mode;
    pb = st.pb;
    scale = st.scale;
  }
  const bool amm = !SETUP && (mode == kPrevious || mode == kProposed);
  const bool centred = !SETUP && mode == kProposed;
  const bool sampled = amm && !a.cc.sanity;
  const int which = centred ? 1 : 0;

  // ---- this CTA's column list -------------------------------------------------------
  int64_t lo = 0, hi = 0;
  if (!sampled) {
    lo = (int64_t)bid * b.n / G;
    hi = (int64_t)(bid + 1) * b.n / G;
  } else {
    // exclusive prefix of the distinct counts per chunk (stage area is scratch here)
    uint32_t* cpre = reinterpret_cast<uint32_t*>(stage_base);
    const uint32_t* chunk = b.chunk[pb];
    uint32_t carry = 0;
    for (int base = 0; base < b.nchunks; base += T) {
      const int k = base + t;
      const uint32_t v = k < b.nchunks ? chunk[k] : 0u;
      uint32_t tot;
      const uint32_t ex = block_exclusive_scan(v, scan, &tot);
      if (k < b.nchunks) cpre[k] = carry + ex;
      carry += tot;
    }
    __syncthreads();
    const uint32_t cd = carry;
    lo = (int64_t)bid * cd / G;
    hi = (int64_t)(bid + 1) * cd / G;
    if (bid == 0 && t == 0) b.distinct_hist[a.iter] = (int32_t)cd;
    if (hi > lo) {
      // chunk holding rank lo: the largest k with cpre[k] <= lo
      int ka = 0, kb = b.nchunks - 1;
      while (ka < kb) {
        const int mid = (ka + kb + 1) >> 1;
        if (cpre[mid] <= (uint32_t)lo)
          ka = mid;
        else
          kb = mid - 1;
      }
      const uint32_t* cnt = b.count[pb];
      const int CH = 1 << b.chunk_shift;
      for (int kc = ka; kc < b.nchunks && cpre[kc] < (uint32_t)hi; ++kc) {
        uint32_t rank0 = cpre[kc];
        const int start = kc << b.chunk_shift;
        const int len = min(CH, b.n - start);
        for (int p0 = 0; p0 < len; p0 += T) {
          const int p = p0 + t;
          const uint32_t mult = p < len ? cnt[start + p] : 0u;
          uint32_t tot;
          const uint32_t ex = block_exclusive_scan(mult ? 1u : 0u, scan, &tot);
          const int64_t r = (int64_t)rank0 + ex;
          if (mult && r >= lo && r < hi) {
            wl_idx[r - lo] = (uint32_t)(start + p);
            wl_mult[r - lo] = mult;
          }
          rank0 += tot;
        }
      }
    }
    __syncthreads();
    for (int k = t; k < (int)(hi - lo); k += T) {
      b.distinct_idx[lo + k] = wl_idx[k];
      b.distinct_mult[lo + k] = wl_mult[k];
    }
  }
  const int nb = (int)(hi - lo);
  const int gc = g.gc, NS = g.nstages;
  const int ngroups = (nb + gc - 1) / gc;
  const uint64_t policy = l2_evict_first_policy();
  const size_t col_stride = (size_t)b.ld * sizeof(Elem);
  const unsigned char* Abase = reinterpret_cast<const unsigned char*>(b.A);

  auto column_of = [&](int k) -> uint32_t {
    return sampled ? wl_idx[k] : (uint32_t)(lo + k);
  };
  auto issue = [&](int grp) {
    const int s = grp % NS;
    const int c0 = grp * gc;
    const int cnt = min(gc, nb - c0);
    mbar_arrive_expect_tx(&bars[s], (uint32_t)(cnt * g.colbytes));
    for (int q = 0; q < cnt; ++q) {
      const uint32_t col = column_of(c0 + q);
      bulk_g2s(stage_base + (size_t)s * g.stage_bytes + (size_t)q * g.colbytes,
               Abase + (size_t)col * col_stride, (uint32_t)g.colbytes, &bars[s], policy);
    }
  };

  if (t == 0) {
    for (int s = 0; s < NS; ++s) mbar_init(&bars[s], 1);
    fence_barrier_init();
  }
  __syncthreads();
  if (t == 0) {
    fence_proxy_async_smem();
    for (int grp = 0; grp < min(NS, ngroups); ++grp) issue(grp);
  }

  // ---- dx = x_i − x_memo in registers (x_i = scale * y_{i-1}, FP32) --------------------
  float dx[R][E];
  float yacc[R][E];
#pragma unroll
  for (int r = 0; r < R; ++r)
#pragma unroll
    for (int e = 0; e < E; ++e) {
      dx[r][e] = 0.f;
      yacc[r][e] = 0.f;
    }
  double sum_dx = 0.0, zdx = 0.0;
  if (!SETUP) {
    const float* yprev = b.y[(a.iter + 1) & 1];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int vi = t + r * T;
      if (vi < nvec) {
#pragma unroll
        for (int h = 0; h < E / 4; ++h) {
          const float4 yp = reinterpret_cast<const float4*>(yprev)[vi * (E / 4) + h];
          float4 xm = make_float4(0.f, 0.f, 0.f, 0.f);
          if (amm) xm = reinterpret_cast<const float4*>(b.x_memo)[vi * (E / 4) + h];
          dx[r][4 * h + 0] = __fsub_rn(__fmul_rn(scale, yp.x), xm.x);
          dx[r][4 * h + 1] = __fsub_rn(__fmul_rn(scale, yp.y), xm.y);
          dx[r][4 * h + 2] = __fsub_rn(__fmul_rn(scale, yp.z), xm.z);
          dx[r][4 * h + 3] = __fsub_rn(__fmul_rn(scale, yp.w), xm.w);
          if (centred) {
            const float4 zz = reinterpret_cast<const float4*>(b.z)[vi * (E / 4) + h];
            sum_dx += (double)dx[r][4 * h + 0] + (double)dx[r][4 * h + 1] +
                      (double)dx[r][4 * h + 2] + (double)dx[r][4 * h + 3];
            zdx = fma((double)dx[r][4 * h + 0], (double)zz.x, zdx);
            zdx = fma((double)dx[r][4 * h + 1], (double)zz.y, zdx);
            zdx = fma((double)dx[r][4 * h + 2], (double)zz.z, zdx);
            zdx = fma((double)dx[r][4 * h + 3], (double)zz.w, zdx);
          }
        }
      }
    }
    if (centred) {  // Σdx and z·dx (common.h:55-87), identical in every CTA
      sum_dx = warp_sum(sum_dx);
      zdx = warp_sum(zdx);
      if (lane == 0) {
        red64[2 * warp] = sum_dx;
        red64[2 * warp + 1] = zdx;
      }
      __syncthreads();
      sum_dx = 0.0;
      zdx = 0.0;
      for (int w = 0; w < nwarps; ++w) {
        sum_dx += red64[2 * w];
        zdx += red64[2 * w + 1];
      }
      __syncthreads();
      if (bid == 0 && t == 0) {
        b.st[a.iter & 1].sum_dx = sum_dx;
        b.st[a.iter & 1].zdx = zdx;
      }
    }
  }
  const float sum_dx_f = (float)sum_dx;
  const float* wts = b.wts[which];

  float sacc = 0.f;     // Σ α_k t_k (proposed)
  double a2acc = 0.0;   // Σ α_j² (set-up)
  bool ok = true;

  for (int grp = 0; grp < ngroups; ++grp) {
    const int s = grp % NS;
    const uint32_t parity = (uint32_t)((grp / NS) & 1);
    const bool mbar_ok = mbar_wait_bounded(&bars[s], parity);
    const int cnt = mbar_ok ? min(gc, nb - grp * gc) : 0;
    const unsigned char* sbuf = stage_base + (size_t)s * g.stage_bytes;
    const bool got = mbar_ok;
    float d[kGcMax];
    double s1[SETUP ? kGcMax : 1], s2[SETUP ? kGcMax : 1];
#pragma unroll
    for (int q = 0; q < kGcMax; ++q) d[q] = 0.f;
#pragma unroll
    for (int q = 0; q < (SETUP ? kGcMax : 1); ++q) {
      s1[q] = 0.0;
      s2[q] = 0.0;
    }
#pragma unroll
    for (int q = 0; q < kGcMax; ++q) {
      if (q < cnt) {
        const uint4* col = reinterpret_cast<const uint4*>(sbuf + (size_t)q * g.colbytes);
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int vi = t + r * T;
          if (vi < nvec) {
            float av[E];
            unpack(col[vi], av);
            if constexpr (SETUP) {
#pragma unroll
              for (int e = 0; e < E; ++e) {
                s1[q] += (double)av[e];
                s2[q] = fma((double)av[e], (double)av[e], s2[q]);
              }
            } else {
#pragma unroll
              for (int e = 0; e < E; ++e) d[q] = fmaf(av[e], dx[r][e], d[q]);
            }
          }
        }
      }
    }
    const int rb = grp & 1;
    if constexpr (SETUP) {
#pragma unroll
      for (int q = 0; q < kGcMax; ++q) {
        if (q < cnt) {
          s1[q] = warp_sum(s1[q]);
          s2[q] = warp_sum(s2[q]);
          if (lane == 0) {
            red64[((rb * 16 + warp) * kGcMax + q) * 2] = s1[q];
            red64[((rb * 16 + warp) * kGcMax + q) * 2 + 1] = s2[q];
          }
        }
      }
    } else {
#pragma unroll
      for (int q = 0; q < kGcMax; ++q) {
        if (q < cnt) {
          d[q] = warp_sum(d[q]);
          if (lane == 0) red[(rb * 16 + warp) * kGcMax + q] = d[q];
        }
      }
    }
    // the barrier also makes a timed-out wait block-uniform
    if (__syncthreads_or(got ? 0 : 1)) {
      ok = false;
      break;
    }
    // refill the stage consumed by the previous group (everyone has finished with it)
    if (t == 0 && grp >= 1 && grp - 1 + NS < ngroups) issue(grp - 1 + NS);
    float coef[kGcMax];
#pragma unroll
    for (int q = 0; q < kGcMax; ++q) {
      coef[q] = 0.f;
      if (q < cnt) {
        const int k = grp * gc + q;
        const uint32_t col = column_of(k);
        if constexpr (SETUP) {
          double ss = 0.0, qq = 0.0;
          for (int w = 0; w < nwarps; ++w) {
            ss += red64[((rb * 16 + w) * kGcMax + q) * 2];
            qq += red64[((rb * 16 + w) * kGcMax + q) * 2 + 1];
          }
          const double mean = ss / (double)m;
          const float af = (float)mean;
          coef[q] = af;
          a2acc = fma((double)af, (double)af, a2acc);
          if (t == 0) {
            b.alpha[col] = af;
            b.norm[col] = (float)sqrt(qq);
            b.normp[col] = (float)sqrt(fmax(qq - mean * mean * (double)m, 0.0));
          }
        } else {
          float tot = 0.f;
          for (int w = 0; w < nwarps; ++w) tot += red[(rb * 16 + w) * kGcMax + q];
          if (!amm) {
            coef[q] = tot;
          } else {
            const float wm = a.cc.sanity ? 1.0f : __fmul_rn(wts[col], (float)wl_mult[k]);
            if (centred) {
              const float al = b.alpha[col];
              const float tq = __fmul_rn(__fsub_rn(tot, __fmul_rn(al, sum_dx_f)), wm);
              coef[q] = tq;
              sacc = fmaf(al, tq, sacc);
            } else {
              coef[q] = __fmul_rn(tot, wm);
            }
          }
        }
      }
    }
#pragma unroll
    for (int q = 0; q < kGcMax; ++q) {
      if (q < cnt) {
        const uint4* col = reinterpret_cast<const uint4*>(sbuf + (size_t)q * g.colbytes);
        const float cq = coef[q];
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int vi = t + r * T;
          if (vi < nvec) {
            float av[E];
            unpack(col[vi], av);
#pragma unroll
            for (int e = 0; e < E; ++e) yacc[r][e] = fmaf(cq, av[e], yacc[r][e]);
          }
        }
      }
    }
  }

  if (!ok) {
    if (t == 0) atomicOr(b.status, (uint32_t)kDevTimeout);
    return;
  }

  float* part = b.partials + (size_t)bid * m;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int vi = t + r * T;
    if (vi < nvec) {
#pragma unroll
      for (int h = 0; h < E / 4; ++h)
        reinterpret_cast<float4*>(part)[vi * (E / 4) + h] =
            make_float4(yacc[r][4 * h], yacc[r][4 * h + 1], yacc[r][4 * h + 2], yacc[r][4 * h + 3]);
    }
  }
  if (t == 0) {
    b.spart[bid] = sacc;
    b.spart64[bid] = a2acc;
  }
}

// ------------------------------------------------------------------------------------------
// Reduce kernels
// ------------------------------------------------------------------------------------------
constexpr int kRedThreads = 256;
constexpr int kRedRows = 128;  // rows per reduce CTA: 32 float4 groups x 8 partial slices

// Deterministic sum over the nsm partials of 4 rows starting at row (FP64, fixed order).
__device__ __forceinline__ void reduce_rows(const Buffers& b, int row, double4 (*red)[32],
                                            double4* out) {
  const int rg = threadIdx.x & 31, ps = threadIdx.x >> 5;
  double4 acc = make_double4(0, 0, 0, 0);
  if (row < b.m) {
    for (int k = ps; k < b.nsm; k += 8) {
      const float4 p = *reinterpret_cast<const float4*>(b.partials + (size_t)k * b.m + row);
      acc.x += p.x;
      acc.y += p.y;
      acc.z += p.z;
      acc.w += p.w;
    }
  }
  red[ps][rg] = acc;
  __syncthreads();
  if (ps == 0) {
    double4 s = red[0][rg];
    for (int k = 1; k < 8; ++k) {
      s.x += red[k][rg].x;
      s.y += red[k][rg].y;
      s.z += red[k][rg].z;
      s.w += red[k][rg].w;
    }
    *out = s;
  }
}

__global__ void __launch_bounds__(kRedThreads) setup_reduce_kernel(const __grid_constant__ Buffers b) {
  __shared__ double4 red[8][32];
  __shared__ double a2s;
  const int t = threadIdx.x;
  if (t < 32) {
    double s = 0.0;
    for (int k = t; k < b.nsm; k += 32) s += b.spart64[k];
    s = warp_sum(s);
    if (t == 0) a2s = s;
  }
  const int row = blockIdx.x * kRedRows + (t & 31) * 4;
  double4 z;
  reduce_rows(b, row, red, &z);
  __syncthreads();
  const double a2 = a2s;
  if (t < 32 && row < b.m) {
    const float4 zf = make_float4((float)z.x, (float)z.y, (float)z.z, (float)z.w);
    *reinterpret_cast<float4*>(b.z + row) = zf;
    *reinterpret_cast<float4*>(b.v + row) =
        make_float4((float)((double)zf.x - a2), (float)((double)zf.y - a2),
                    (float)((double)zf.z - a2), (float)((double)zf.w - a2));
  }
  if (blockIdx.x == 0 && t == 0) *b.alpha2 = a2;
}

struct ReduceArgs {
  Buffers b;
  CallCfg cc;
  int iter;
  int nred;
};

__global__ void __launch_bounds__(kRedThreads) reduce_kernel(const __grid_constant__ ReduceArgs a) {
  const Buffers& b = a.b;
  const CallCfg& cc = a.cc;
  const int t = threadIdx.x;
  const IterState st = b.st[a.iter & 1];
  IterState* st_next = &b.st[(a.iter + 1) & 1];
  if (st.done) {
    if (blockIdx.x == 0 && t == 0) *st_next = st;
    return;
  }
  const bool consumed = (st.mode == kPrevious || st.mode == kProposed);

  if ((int)blockIdx.x >= a.nred) {
    // draw the picks of the next AMM step while the sums are reduced
    if (consumed && !cc.sanity) {
      const int which = next_amm_weighting(cc, a.iter);
      sampling_role(b, which, st.pb, st.sb ^ 1, st.pb ^ 1, blockIdx.x - a.nred,
                    gridDim.x - a.nred, a.iter + 1 < cc.step);
    }
    return;
  }

  __shared__ double4 red[8][32];
  __shared__ double s_shared;
  __shared__ int is_last;
  if (t < 32) {
    double s = 0.0;
    if (st.mode == kProposed)
      for (int k = t; k < b.nsm; k += 32) s += (double)b.spart[k];
    s = warp_sum(s);
    if (t == 0) s_shared = s;
  }
  const int row = blockIdx.x * kRedRows + (t & 31) * 4;
  double4 tot;
  reduce_rows(b, row, red, &tot);
  __syncthreads();
  if (t < 32) {
    double xy = 0.0, yy = 0.0, yv = 0.0;
    if (row < b.m) {
      const float* yprev = b.y[(a.iter + 1) & 1];
      const float4 yp = *reinterpret_cast<const float4*>(yprev + row);
      const float4 xi = make_float4(__fmul_rn(st.scale, yp.x), __fmul_rn(st.scale, yp.y),
                                    __fmul_rn(st.scale, yp.z), __fmul_rn(st.scale, yp.w));
      double tv[4] = {tot.x, tot.y, tot.z, tot.w};
      float yo[4];
      const float xa[4] = {xi.x, xi.y, xi.z, xi.w};
      if (st.mode == kExact || st.mode == kExactMemo) {
#pragma unroll
        for (int e = 0; e < 4; ++e) yo[e] = (float)tv[e];
      } else {
        const float4 ym = *reinterpret_cast<const float4*>(b.y_memo + row);
        const float ymv[4] = {ym.x, ym.y, ym.z, ym.w};
        if (st.mode == kPrevious) {
#pragma unroll
          for (int e = 0; e < 4; ++e) yo[e] = (float)((double)ymv[e] + tv[e]);
        } else {
          // y_memo + Σdx·v + z·dx in FP64, rounded (core_proposedAMM.cuh:198-212)
          const float4 vv = *reinterpret_cast<const float4*>(b.v + row);
          const float va[4] = {vv.x, vv.y, vv.z, vv.w};
          const double S = s_shared;
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const float base = (float)(fma(st.sum_dx, (double)va[e], st.zdx) + (double)ymv[e]);
            yo[e] = (float)((double)base + (tv[e] - S));
          }
        }
      }
      *reinterpret_cast<float4*>(b.y[a.iter & 1] + row) = make_float4(yo[0], yo[1], yo[2], yo[3]);
      if (st.mode == kExactMemo) {
        *reinterpret_cast<float4*>(b.x_memo + row) = xi;
        *reinterpret_cast<float4*>(b.y_memo + row) = make_float4(yo[0], yo[1], yo[2], yo[3]);
      }
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const double yd = (double)yo[e];
        xy = fma(yd, (double)xa[e], xy);
        yy = fma(yd, yd, yy);
        if (b.has_vstar) yv = fma(yd, b.vstar[row + e], yv);
      }
    }
    xy = warp_sum(xy);
    yy = warp_sum(yy);
    yv = warp_sum(yv);
    if (t == 0) {
      b.rpart[4 * blockIdx.x + 0] = xy;
      b.rpart[4 * blockIdx.x + 1] = yy;
      b.rpart[4 * blockIdx.x + 2] = yv;
      __threadfence();
      const uint32_t old = atomicAdd(&b.ticket[0], 1u);
      is_last = (old == (uint32_t)(a.nred - 1));
    }
  }
  __syncthreads();
  if (!is_last || t != 0) return;
  __threadfence();
  // last CTA: Rayleigh quotient and the next step (common.h:103-153)
  double xy = 0.0, yy = 0.0, yv = 0.0;
  const volatile double* rp = b.rpart;
  for (int k = 0; k < a.nred; ++k) {
    xy += rp[4 * k + 0];
    yy += rp[4 * k + 1];
    yv += rp[4 * k + 2];
  }
  b.ticket[0] = 0u;
  const double scale = rsqrt(yy);
  const double lam = xy;
  const double err = yv * scale;
  const double cosv = lam * scale;
  const int i = a.iter;
  b.eigs[i] = lam;
  b.errs[i] = err;
  b.coss[i] = cosv;
  b.kinds[i] = st.mode;
  if (!consumed || cc.sanity) b.distinct_hist[i] = b.n;
  b.tstamp[i + 1] = globaltimer_ns();
  IterState nx = st;
  nx.scale = (float)scale;
  nx.cos_prev = cosv;
  nx.lam_prev = lam;
  nx.steps_run = i + 1;
  if (consumed && !cc.sanity) {
    nx.sb = st.sb ^ 1;
    nx.pb = st.pb ^ 1;
  }
  bool done = false;
  if (!isfinite(lam) || !isfinite(scale)) {
    atomicOr(b.status, (uint32_t)kDevNonFinite);
    done = true;
  }
  if (cc.tol > 0.0 && i >= 1 && fabs(lam - st.lam_prev) <= cc.tol * fabs(lam)) done = true;
  nx.done = done ? 1 : 0;
  int le;
  nx.mode = decide_mode(cc, i + 1, cosv, st.last_exact, &le);
  nx.last_exact = le;
  *st_next = nx;
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

__global__ void __launch_bounds__(kRedThreads) init_kernel(const __grid_constant__ InitArgs a) {
  const Buffers& b = a.b;
  const CallCfg& cc = a.cc;
  const int t = threadIdx.x;
  if (blockIdx.x > 0) {
    if (cc.uses_amm && !cc.sanity)
      sampling_role(b, next_amm_weighting(cc, -1), -1, 0, 0, blockIdx.x - 1, gridDim.x - 1, true);
    return;
  }
  __shared__ double ws[kRedThreads / 32];
  double ss = 0.0;
  for (int k = t; k < b.m; k += blockDim.x) {
    const float v = a.x0[k];
    b.y[1][k] = v;
    ss = fma((double)v, (double)v, ss);
  }
  ss = warp_sum(ss);
  if ((t & 31) == 0) ws[t >> 5] = ss;
  __syncthreads();
  if (t == 0) {
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
    st.sb = 0;
    st.pb = 0;
    st.steps_run = 0;
    if (!(s > 0.0) || !isfinite(s)) {
      atomicOr(b.status, (uint32_t)kDevNonFinite);
      st.done = 1;
    }
    b.st[0] = st;
    b.tstamp[0] = globaltimer_ns();
  }
}

struct FinalArgs {
  Buffers b;
  CallCfg cc;
  float* xdst;
  float* ydst;
};

__global__ void __launch_bounds__(kRedThreads) finalize_kernel(const __grid_constant__ FinalArgs a) {
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
  if (a.cc.uses_amm && !a.cc.sanity) {
    if (st.sb == 1)
      for (int k = gt; k < b.c; k += gs) b.states[0][k] = b.states[1][k];
    // pending (speculative) picks are dropped: their states were never committed
    uint32_t* cnt = b.count[st.pb];
    const uint32_t* smp = b.samples[st.pb];
    for (int k = gt; k < b.c; k += gs) cnt[smp[k]] = 0u;
    for (int k = gt; k < b.nchunks; k += gs) b.chunk[st.pb][k] = 0u;
  }
}

// ------------------------------------------------------------------------------------------
// CDF construction (once per matrix)
// ------------------------------------------------------------------------------------------
constexpr int kCdfThreads = 1024;
constexpr int kCdfTile = 4096;

// blockIdx.x selects the weighting (or `which` when >= 0).  FP64 mode: weight_j =
// (double)norm_j², CDF = FP64 inclusive prefix.  FP32 mode: weight_j = fl32(norm_j²) as
// set_weights (common.h:34-40); CDF = fl32 of the FP64 prefix of those weights.  Then
// w_j = total/(weight_j·c) (update_weights, common.h:42-53) and the coarse table.
__global__ void __launch_bounds__(kCdfThreads) build_cdf_kernel(const __grid_constant__ Buffers b,
                                                                int which_in, int keep_cdf,
                                                                int sanity) {
  __shared__ double tile[kCdfTile];
  __shared__ double wsum[32];
  __shared__ double carry_s;
  const int which = which_in >= 0 ? which_in : (int)blockIdx.x;
  const float* base = which == 0 ? b.norm : b.normp;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int n = b.n;
  constexpr int PER = kCdfTile / kCdfThreads;
  if (!keep_cdf) {
    double carry = 0.0;
    for (int t0 = 0; t0 < n; t0 += kCdfTile) {
      for (int k = t; k < kCdfTile; k += kCdfThreads) {
        const int j = t0 + k;
        double w = 0.0;
        if (j < n) {
          const float nv = base[j];
          w = sanity ? 1.0 : (b.cdf_f32 ? (double)__fmul_rn(nv, nv) : (double)nv * (double)nv);
        }
        tile[k] = w;
      }
      __syncthreads();
      double loc = 0.0;
#pragma unroll
      for (int e = 0; e < PER; ++e) loc += tile[t * PER + e];
      double incl = loc;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const double y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
      }
      if (lane == 31) wsum[warp] = incl;
      __syncthreads();
      if (warp == 0) {
        const double w = wsum[lane];
        double wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const double y = __shfl_up_sync(0xffffffffu, wi, o);
          if (lane >= o) wi += y;
        }
        wsum[lane] = wi - w;
        if (lane == 31) carry_s = wi;
      }
      __syncthreads();
      double run = carry + wsum[warp] + (incl - loc);
#pragma unroll
      for (int e = 0; e < PER; ++e) {
        const int j = t0 + t * PER + e;
        run += tile[t * PER + e];
        if (j < n) {
          if (b.cdf_f32)
            b.cdf32[which][j] = (float)run;
          else
            b.cdf64[which][j] = run;
        }
      }
      carry += carry_s;
      __syncthreads();
    }
  }
  __syncthreads();
  const double total64 = b.cdf_f32 ? (double)b.cdf32[which][n - 1] : b.cdf64[which][n - 1];
  const float total32 = b.cdf_f32 ? b.cdf32[which][n - 1] : (float)total64;
  for (int j = t; j < n; j += kCdfThreads) {
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
  for (int s = t; s < b.ncoarse; s += kCdfThreads) {
    const int j = (s + 1) * b.seg - 1;
    if (b.cdf_f32)
      b.coarse32[which][s] = b.cdf32[which][j];
    else
      b.coarse64[which][s] = b.cdf64[which][j];
  }
  if (t == 0 && (!(total64 > 0.0) || !isfinite(total64)))
    atomicOr(b.status, (uint32_t)kDevNonFinite);
}

// ------------------------------------------------------------------------------------------
// Standalone helpers (not on the iteration path)
// ------------------------------------------------------------------------------------------
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
bool panel_geometry(int m, int dtype, int c, int n, int nsm, PanelGeom* g) {
  const int es = dtype == 1 ? 2 : 4;
  const int E = 16 / es;
  if (m <= 0 || m % E != 0) return false;
  const int nvec = m / E;
  int R = 1;
  while (R < 8 && (nvec + R - 1) / R > kMaxThreads) R <<= 1;
  if ((nvec + R - 1) / R > kMaxThreads) return false;
  if (R * E > 32) return false;  // register budget: 32 rows per thread
  int threads = ((nvec + R - 1) / R + 31) / 32 * 32;
  g->threads = threads;
  g->slots = R;
  g->elems = E;
  g->colbytes = m * es;
  const int budget = 200 * 1024;
  int target_stage = 48 * 1024;
  int gc = target_stage / g->colbytes;
  if (gc < 1) gc = 1;
  if (gc > kGcMax) gc = kGcMax;
  int stage = gc * g->colbytes;
  int ns = budget / stage;
  if (ns > 6) ns = 6;
  if (ns < 2) {
    ns = 2;
    gc = 1;
    stage = g->colbytes;
    if (2 * stage > budget) return false;
  }
  g->gc = gc;
  g->nstages = ns;
  g->stage_bytes = stage;
  int maxlist = c < n ? c : n;
  int wl = (maxlist + nsm - 1) / nsm + 1;
  g->wl_cap = wl;
  // the stage area doubles as scratch for the per-chunk prefix (<= 4096 uint32) before the
  // pipeline starts
  g->stage_area = ns * stage > 4 * 4096 ? ns * stage : 4 * 4096;
  g->smem_bytes = g->stage_area + 8 * 8 + 4096 + 2 * wl * 4 + 40 * 4;
  return g->smem_bytes <= 227 * 1024;
}

template <typename Elem, int R>
static cudaError_t launch_panel_t(const PanelArgs& a, cudaStream_t s) {
  auto k = a.setup ? panel_kernel<Elem, R, true> : panel_kernel<Elem, R, false>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       a.g.smem_bytes);
  if (e != cudaSuccess) return e;
  k<<<a.b.nsm, a.g.threads, a.g.smem_bytes, s>>>(a);
  count_launch();
  return cudaGetLastError();
}

static cudaError_t launch_panel(const PanelArgs& a, cudaStream_t s) {
  const bool bf = a.b.dtype == 1;
  switch (a.g.slots) {
    case 1: return bf ? launch_panel_t<__nv_bfloat16, 1>(a, s) : launch_panel_t<float, 1>(a, s);
    case 2: return bf ? launch_panel_t<__nv_bfloat16, 2>(a, s) : launch_panel_t<float, 2>(a, s);
    case 4: return bf ? launch_panel_t<__nv_bfloat16, 4>(a, s) : launch_panel_t<float, 4>(a, s);
    case 8: return launch_panel_t<float, 8>(a, s);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_setup_panel(const Buffers& b, const PanelGeom& g, cudaStream_t s) {
  PanelArgs a{};
  a.b = b;
  a.g = g;
  a.iter = 0;
  a.setup = 1;
  return launch_panel(a, s);
}

cudaError_t launch_iter_panel(const Buffers& b, const PanelGeom& g, const CallCfg& cc, int iter,
                              cudaStream_t s) {
  PanelArgs a{};
  a.b = b;
  a.g = g;
  a.cc = cc;
  a.iter = iter;
  a.setup = 0;
  return launch_panel(a, s);
}

static int reduce_ctas(int m) { return (m + kRedRows - 1) / kRedRows; }
static int sample_ctas(int c) {
  int k = (c + kRedThreads * 4 - 1) / (kRedThreads * 4);
  return k < 1 ? 1 : (k > 64 ? 64 : k);
}

cudaError_t launch_setup_reduce(const Buffers& b, cudaStream_t s) {
  setup_reduce_kernel<<<reduce_ctas(b.m), kRedThreads, 0, s>>>(b);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_build_cdf(const Buffers& b, int which, int keep_cdf, int sanity,
                             cudaStream_t s) {
  build_cdf_kernel<<<which >= 0 ? 1 : 2, kCdfThreads, 0, s>>>(b, which, keep_cdf, sanity);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_init(const Buffers& b, const CallCfg& cc, const float* x0, int no_normalize,
                        cudaStream_t s) {
  InitArgs a{};
  a.b = b;
  a.cc = cc;
  a.x0 = x0;
  a.no_normalize = no_normalize;
  const int ns = (cc.uses_amm && !cc.sanity) ? sample_ctas(b.c) : 0;
  init_kernel<<<1 + ns, kRedThreads, 0, s>>>(a);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_iter_reduce(const Buffers& b, const CallCfg& cc, int iter, cudaStream_t s) {
  ReduceArgs a{};
  a.b = b;
  a.cc = cc;
  a.iter = iter;
  a.nred = reduce_ctas(b.m);
  const int ns = (cc.uses_amm && !cc.sanity) ? sample_ctas(b.c) : 0;
  reduce_kernel<<<a.nred + ns, kRedThreads, 0, s>>>(a);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_finalize(const Buffers& b, const CallCfg& cc, float* xdst, float* ydst,
                            cudaStream_t s) {
  FinalArgs a{};
  a.b = b;
  a.cc = cc;
  a.xdst = xdst;
  a.ydst = ydst;
  int blocks = (b.m + kRedThreads - 1) / kRedThreads;
  if (blocks > 256) blocks = 256;
  finalize_kernel<<<blocks, kRedThreads, 0, s>>>(a);
  count_launch();
  return cudaGetLastError();
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
