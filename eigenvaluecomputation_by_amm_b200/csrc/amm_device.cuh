// Device helpers shared by the kernels of libamm (PTX wrappers for mbarriers, bulk copies and
// distributed shared memory; warp/block reductions; BF16 unpacking).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "amm_internal.h"

namespace amm {

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

__device__ __forceinline__ unsigned long long globaltimer_now() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

// Upper bound of every device-side wait of this library: after it the wait gives up, the
// caller records kDevTimeout and winds down, so a kernel never spins without end.
constexpr unsigned long long kWaitLimitNs = 2000000000ull;

// Bounded wait on an mbarrier phase (CTA scope): false after kWaitLimitNs.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = globaltimer_now();
  for (uint32_t it = 1;; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((it & 255u) == 0 && globaltimer_now() - t0 > kWaitLimitNs) return false;
  }
}

// Asynchronous global -> shared copies of 4 and 16 bytes (no register staging: the issuing
// thread goes on and waits only at cp_async_wait_all).
__device__ __forceinline__ void cp_async4(void* smem_dst, const void* gsrc) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_addr(smem_dst)), "l"(gsrc)
               : "memory");
}
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gsrc) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(smem_dst)), "l"(gsrc)
               : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
// 16-byte copy of which only the first src_bytes (0..16) are read; the rest of the destination
// is zero-filled (src must still be a valid 16-byte aligned address)
__device__ __forceinline__ void cp_async16_zfill(void* smem_dst, const void* gsrc, int src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_addr(smem_dst)),
               "l"(gsrc), "r"(src_bytes)
               : "memory");
}
// 2-D tensor copy (TMA) of one box at element coordinates (x, y) of the tensor map at `tmap`
// (global memory) into this CTA's shared memory, completing bytes on `bar` (complete_tx).  x is
// the innermost coordinate; x times the element size must be a multiple of 16 bytes.
__device__ __forceinline__ void tma_load_2d(void* smem_dst, const void* tmap, int x, int y,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_addr(smem_dst)),
      "l"(tmap), "r"(x), "r"(y), "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// waits until at most N of this thread's committed copy groups are still in flight
template <int N>
__device__ __forceinline__ void cp_async_wait_group() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
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


// ---- thread-block clusters and distributed shared memory ----
__device__ __forceinline__ uint32_t cluster_ctarank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t cluster_nctarank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
  return r;
}
// Address of the same shared-memory location in CTA `rank` of this cluster.
__device__ __forceinline__ uint32_t map_to_rank(uint32_t local_addr, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(local_addr), "r"(rank));
  return r;
}
__device__ __forceinline__ void st_cluster_f32(uint32_t addr, float v) {
  asm volatile("st.shared::cluster.f32 [%0], %1;" ::"r"(addr), "f"(v) : "memory");
}
__device__ __forceinline__ void st_cluster_f64(uint32_t addr, double v) {
  asm volatile("st.shared::cluster.f64 [%0], %1;" ::"r"(addr), "d"(v) : "memory");
}
// Arrive (release, cluster scope) on an mbarrier given by its cluster-mapped address.
__device__ __forceinline__ void mbar_arrive_remote(uint32_t cluster_addr) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(cluster_addr)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive_local(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}
// try_wait with acquire at cluster scope (data written by peers before their release-arrive).
__device__ __forceinline__ bool mbar_try_wait_cluster(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_cluster_bounded(uint64_t* bar, uint32_t parity) {
  if (mbar_try_wait_cluster(bar, parity)) return true;
  const unsigned long long t0 = globaltimer_now();
  for (uint32_t it = 1;; ++it) {
    if (mbar_try_wait_cluster(bar, parity)) return true;
    if ((it & 255u) == 0 && globaltimer_now() - t0 > kWaitLimitNs) return false;
  }
}
// 16-byte load from shared memory given by its cluster-mapped address (a peer CTA's included).
__device__ __forceinline__ float4 ld_cluster_f4(uint32_t cluster_addr) {
  float4 v;
  asm volatile("ld.shared::cluster.v4.f32 {%0, %1, %2, %3}, [%4];"
               : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
               : "r"(cluster_addr)
               : "memory");
  return v;
}
// Orders this thread's earlier memory accesses before its later ones at cluster scope.
__device__ __forceinline__ void fence_acq_rel_cluster() {
  asm volatile("fence.acq_rel.cluster;" ::: "memory");
}
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release;\n\tbarrier.cluster.wait.acquire;" ::: "memory");
}
// Named barrier over `nthreads` threads with an OR-reduction of `pred` (block-uniform result).
__device__ __forceinline__ bool named_barrier_or(int id, int nthreads, bool pred) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.or.pred q, %2, %3, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}"
      : "=r"(r)
      : "r"((uint32_t)pred), "r"(id), "r"(nthreads)
      : "memory");
  return r != 0;
}

// ---- the reference's random draw (get_rand, device_memory.h:506-514) ----
__device__ __forceinline__ uint32_t xorshift32(uint32_t y) {
  y ^= (y << 13);
  y ^= (y >> 17);
  y ^= (y << 5);
  return y;
}
// exact: 1.mantissa - 1 (device_memory.h:513)
__device__ __forceinline__ float uniform_from(uint32_t y) {
  return __fsub_rn(__uint_as_float((y & 0x007FFFFFu) | 0x3f800000u), 1.0f);
}

// Kind of the step that follows, as the reference's drivers decide it:
//  previous    powerMethod_by_previous.cuh:135-137
//  proposed    powerMethod_by_proposed.cuh:371-373 (no VR right after a VR step)
//  proposed_v2 powerMethod_by_proposed_v2.cuh:234-305
__device__ __forceinline__ int decide_mode(const CallCfg& cc, int i, double cos_prev, int last_exact,
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

// Weighting (0 = ‖A_j‖², 1 = ‖A_j − α_j‖²) of a call's AMM step number `list` (0-based count of
// the steps that consume picks): the proposed_v2 driver samples with ‖A_j‖² during its
// previous-AMM warm-up (steps 0 .. vr_period-2) and with ‖A_j − α_j‖² after its exact step.
__device__ __forceinline__ int list_weighting(const CallCfg& cc, int list) {
  if (cc.method == kMethodPrevious) return 0;
  if (cc.method == kMethodProposed) return 1;
  if (cc.method == kMethodProposedV2) return list < cc.vr_period - 1 ? 0 : 1;
  return 0;
}

// End of the work lists drawn once the window is refilled ahead of step i (i % kListWindow ==
// 0), from the state that step i starts with: the next kListWindow AMM steps, but no more than
// the steps left in the call; lists already drawn stay (pending lists are never redrawn).
__host__ __device__ __forceinline__ int32_t window_end(const CallCfg& cc, int i,
                                                       const IterState& st) {
  const int32_t left = cc.step - i;
  const int32_t e = st.used + (left < kListWindow ? left : kListWindow);
  return e > st.drawn ? e : st.drawn;
}

// The step's scalars from the summed x·y, y·y and y·v* (dotProduct_and_generate_x,
// common.h:103-153): λ = x·y, err = y·v*/‖y‖, cos = λ/‖y‖, and the state of the next step (its
// scale, its kind, the tolerance stop).  A pure function of its arguments: every CTA of the
// step kernel evaluates it on the same sums and gets the same state.
struct StepScalars {
  double lam, err, cosv;
  bool nonfinite;
};

__device__ __forceinline__ IterState next_state(const CallCfg& cc, int i, const IterState& st,
                                                double xy, double yy, double yv,
                                                StepScalars* sc) {
  const bool consumed = st.mode == kPrevious || st.mode == kProposed;
  const double scale = rsqrt(yy);
  const double lam = xy;
  sc->lam = lam;
  sc->err = yv * scale;
  sc->cosv = lam * scale;
  IterState nx = st;
  nx.scale = (float)scale;
  nx.cos_prev = sc->cosv;
  nx.lam_prev = lam;
  nx.steps_run = i + 1;
  if (consumed && !cc.sanity) nx.used = st.used + 1;
  if (st.mode == kExactMemo) nx.memo_zero = 0;  // this step wrote the memo pair
  if (cc.uses_amm && !cc.sanity && i % kListWindow == 0) nx.drawn = window_end(cc, i, st);
  sc->nonfinite = !isfinite(lam) || !isfinite(scale);
  bool done = sc->nonfinite;
  if (cc.tol > 0.0 && i >= 1 && fabs(lam - st.lam_prev) <= cc.tol * fabs(lam)) done = true;
  nx.done = done ? 1 : 0;
  int le;
  nx.mode = decide_mode(cc, i + 1, sc->cosv, st.last_exact, &le);
  nx.last_exact = le;
  return nx;
}

// The trace entries of step i (one thread of the grid).
__device__ __forceinline__ void record_step(const Buffers& b, const CallCfg& cc, int i,
                                            const IterState& st, const StepScalars& sc) {
  const bool consumed = st.mode == kPrevious || st.mode == kProposed;
  b.eigs[i] = sc.lam;
  b.errs[i] = sc.err;
  b.coss[i] = sc.cosv;
  b.kinds[i] = st.mode;
  if (!consumed || cc.sanity) b.distinct_hist[i] = b.n;
  b.tstamp[i + 1] = globaltimer_now();
  if (sc.nonfinite) atomicOr(b.status, (uint32_t)kDevNonFinite);
}

// ---- programmatic dependent launch (a grid launched with programmatic stream serialization
// may start while the grid before it in the stream finishes) ----
// Wait until the preceding grid has completed and its memory is visible (returns at once for
// a grid launched without the attribute).
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
// Allow the next grid in the stream to be scheduled (its CTAs take SMs as this grid's retire).
__device__ __forceinline__ void griddep_launch_dependents() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// ---- grid-wide barrier over co-resident CTAs ----
__device__ __forceinline__ uint32_t ld_acquire_gpu(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Called by one thread per CTA after the CTA's own writes are ordered before it (a CTA barrier).
// bar counts arrivals without reset (a call's first kernel zeroes it); every launch adds exactly
// nblocks arrivals, so a barrier completes when the count reaches the next multiple of nblocks.
// Every CTA of the grid must be resident at once (one per SM).  Bounded: returns false if the
// count did not reach the target within kWaitLimitNs.
__device__ __forceinline__ bool grid_barrier(uint32_t* bar, uint32_t nblocks) {
  __threadfence();
  const uint32_t old = atomicAdd(bar, 1u);
  const uint32_t target = (old / nblocks + 1u) * nblocks;
  const unsigned long long t0 = globaltimer_now();
  for (uint32_t it = 0;; ++it) {
    if ((int32_t)(ld_acquire_gpu(bar) - target) >= 0) break;
    if ((it & 31u) == 31u && globaltimer_now() - t0 > kWaitLimitNs) return false;
    __nanosleep(20);
  }
  __threadfence();
  return true;
}

// Warp reduction of N values at once (multi-value butterfly): lane l ends with the full sum of
// value l / (32/N); returns it (a fixed tree, deterministic).
template <typename V, int N>
__device__ __forceinline__ V warp_reduce_multi(V (&v)[N], int lane) {
  int off = 16;
#pragma unroll
  for (int n = N / 2; n >= 1; n >>= 1, off >>= 1) {
    const bool upper = (lane & off) != 0;
#pragma unroll
    for (int i = 0; i < n; ++i) {
      const V send = upper ? v[i] : v[i + n];
      const V keep = upper ? v[i + n] : v[i];
      v[i] = keep + __shfl_xor_sync(0xffffffffu, send, off);
    }
  }
  V r = v[0];
  for (; off > 0; off >>= 1) r += __shfl_xor_sync(0xffffffffu, r, off);
  return r;
}

}  // namespace amm
