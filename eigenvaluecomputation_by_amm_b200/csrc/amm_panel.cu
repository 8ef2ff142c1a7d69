// The fused single-pass product kernel of libamm (sm_100a):
//
//   y_part = Σ_{k in this CTA's columns} coef_k · A_k,   coef_k = f(A_kᵀ·dx)
//
// for one power-method step (all n columns for an exact step, the distinct sampled columns for
// an AMM step) and for the set-up pass (coef_j = α_j, plus FP64 column statistics).
//
// One persistent CTA per SM owns a contiguous range of the column list and all m rows.  Thread 0
// streams the columns, GC per group, into a ring of NS shared-memory stages with 1-D TMA bulk
// copies (mbarrier complete_tx; measured on B200: >= 64 KB in flight per SM saturates HBM),
// refilling a stage once every thread is past it.  All warps hold dx and their share of y in
// registers; per group they
//   1. form the coefficients of group g from the warp partials published at the last barrier,
//   2. compute the partial dots of group g+1 (their rows),
//   3. accumulate coef·A_k of group g into y (packed FP32x2 FMAs),
//   4. warp-reduce and publish the dots of g+1, then meet at one named barrier,
// so the reduction latency of a group hides behind the next group's math and there is one
// barrier per group.  Each column is read from HBM once (the reference's kernel1/kernel2 read
// it twice).  Each CTA writes one partial y (with thread-block clusters, the cluster's CTAs first
// sum theirs through distributed shared memory and write one partial per cluster); after a grid
// barrier every CTA sums its rows of the partials in a fixed order, and every CTA forms λ and
// the next step's state from the same per-CTA sums.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>

#include "amm_device.cuh"
#include "amm_internal.h"

namespace amm {

// column groups of the next step issued at the end of a step's last group
constexpr int kPrefetchGroups = 2;
// CTAs of a persistent grid at most (one per SM): the per-CTA scalars of a step are staged
// in shared memory, 2 per CTA
constexpr int kMaxGrid = 256;
// dynamic shared memory a CTA may use: the opt-in maximum less room for the kernel's static
// shared variables
constexpr int kSmemBudget = 227 * 1024 - 1024;

struct PanelArgs {
  Buffers b;
  PanelGeom g;
  CallCfg cc;
  int iter;      // first step of the launch
  int iter_end;  // steps [iter, iter_end) run in this launch (the set-up pass: one pass)
};

template <bool SETUP>
struct RedT {
  using T = float;
};
template <>
struct RedT<true> {
  using T = double2;  // (Σa, Σa²)
};

__device__ __forceinline__ float red_add(float a, float b) { return a + b; }
__device__ __forceinline__ double2 red_add(double2 a, double2 b) {
  return make_double2(a.x + b.x, a.y + b.y);
}
__device__ __forceinline__ float red_zero(float) { return 0.f; }
__device__ __forceinline__ double2 red_zero(double2) { return make_double2(0.0, 0.0); }
__device__ __forceinline__ float warp_red(float v) { return warp_sum(v); }
__device__ __forceinline__ double2 warp_red(double2 v) {
  return make_double2(warp_sum(v.x), warp_sum(v.y));
}

// Shared memory carve (byte offsets), identical on host and device.
struct SmemLayout {
  int stages, bars, redw, wl_idx, wl_w, wl_al, nxt, red, epi, scal, total;
};

__host__ __device__ inline SmemLayout smem_layout(const PanelGeom& g, bool setup) {
  SmemLayout L{};
  const int rsz = setup ? 16 : 4;
  int o = 0;
  L.stages = o;
  o += g.stage_area;
  L.bars = o;  // full[8]
  o += 8 * 16;
  L.redw = o;  // [2][16 warps][GC]; also 16 x 2 doubles of prologue scratch
  int rw = 2 * 16 * g.gc * rsz;
  if (rw < 16 * 16) rw = 16 * 16;
  o += rw;
  L.wl_idx = o;
  o += 4 * g.wl_cap;
  L.wl_w = o;
  o += 4 * g.wl_cap;
  L.wl_al = o;
  o += 4 * g.wl_cap;
  o = (o + 127) & ~127;
  L.nxt = o;  // first column indices of the next step's list: [kGcMax * 8]
  o += 4 * kGcMax * 8;
  L.red = o;  // row-reduction scratch: [16 warps][32] double4
  o += 16 * 32 * 32;
  L.epi = o;  // this CTA's first 32 row groups of y_{i-1}, y_memo, v, x_memo, z (float4)
  o += 5 * 32 * 16 + 32 * 32;  // and v* (4 doubles)
  L.scal = o;  // the per-CTA scalars of the step (Σ α_k t_k or Σ α_j², z·dx): [2][kMaxGrid]
  o += 2 * kMaxGrid * 8;
  L.total = (o + 127) & ~127;
  return L;
}

// Packed FP32x2 arithmetic (Blackwell): two IEEE-rounded FMAs per instruction (the sm_100
// builtin, so the compiler allocates the register pairs itself).
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

// 16-byte vector -> E/2 float2 (exact for BF16: the 16 bits become the high half).
__device__ __forceinline__ void unpack2(const uint4& v, float2 (&o)[2]) {
  o[0] = make_float2(__uint_as_float(v.x), __uint_as_float(v.y));
  o[1] = make_float2(__uint_as_float(v.z), __uint_as_float(v.w));
}
__device__ __forceinline__ void unpack2(const uint4& v, float2 (&o)[4]) {
  o[0] = make_float2(__uint_as_float(v.x << 16), __uint_as_float(v.x & 0xffff0000u));
  o[1] = make_float2(__uint_as_float(v.y << 16), __uint_as_float(v.y & 0xffff0000u));
  o[2] = make_float2(__uint_as_float(v.z << 16), __uint_as_float(v.z & 0xffff0000u));
  o[3] = make_float2(__uint_as_float(v.w << 16), __uint_as_float(v.w & 0xffff0000u));
}

// Branch-free body of one full group: the axpy of group g (stage `cur`, coefficients `coef`)
// interleaved, slot by slot, with the partial dots of group g+1 (stage `nxt`) when NEXT.  Used
// when every column of both groups is present and every vector slot of every thread is valid.
template <typename Elem, int R, int GC, bool NEXT, int TC>
__device__ __forceinline__ void fused_block(const unsigned char* cur, const unsigned char* nxt,
                                            uint32_t col_bytes, int t, int T_rt,
                                            const float (&coef)[GC],
                                            const float2 (&dx)[R][8 / sizeof(Elem)],
                                            float2 (&yacc)[R][8 / sizeof(Elem)], float (&dn)[GC]) {
  constexpr int H = 8 / sizeof(Elem);
  // with a compile-time thread count (TC > 0) every shared-memory load uses an immediate offset
  const int T = TC > 0 ? TC : T_rt;
  const int colv = TC > 0 ? R * TC : (int)(col_bytes >> 4);  // vectors per column
  const uint4* c4 = reinterpret_cast<const uint4*>(cur) + t;
  const uint4* n4 = reinterpret_cast<const uint4*>(nxt) + t;
  float2 p[GC];
#pragma unroll
  for (int qq = 0; qq < GC; ++qq) p[qq] = make_float2(0.f, 0.f);
#pragma unroll
  for (int r = 0; r < R; ++r) {
    uint4 vc[GC], vn[GC];
#pragma unroll
    for (int qq = 0; qq < GC; ++qq) {
      vc[qq] = c4[qq * colv + r * T];
      if (NEXT) vn[qq] = n4[qq * colv + r * T];
    }
#pragma unroll
    for (int qq = 0; qq < GC; ++qq) {
      float2 ac[H];
      unpack2(vc[qq], ac);
      const float2 c2 = make_float2(coef[qq], coef[qq]);
#pragma unroll
      for (int h = 0; h < H; ++h) yacc[r][h] = fma2(c2, ac[h], yacc[r][h]);
      if (NEXT) {
        float2 an[H];
        unpack2(vn[qq], an);
#pragma unroll
        for (int h = 0; h < H; ++h) p[qq] = fma2(an[h], dx[r][h], p[qq]);
      }
    }
  }
#pragma unroll
  for (int qq = 0; qq < GC; ++qq) dn[qq] = p[qq].x + p[qq].y;
}

// Sum over the 16 warps of NC partial values per warp (element (w, c) at base[w * stride + c]),
// computed identically by every warp: lane groups of L lanes own one value each and reduce by a
// fixed xor tree (deterministic).
template <typename V, int NC>
__device__ __forceinline__ void warp_partials_sum(const V* base, int stride, int lane,
                                                  V (&tot)[NC]) {
  constexpr int L = (32 / NC) < 16 ? (32 / NC) : 16;  // lanes per value
  constexpr int PER = 16 / L;                          // warp partials per lane
  constexpr int CPR = 32 / L;                          // values per round
  constexpr int ROUNDS = (NC + CPR - 1) / CPR;
#pragma unroll
  for (int rr = 0; rr < ROUNDS; ++rr) {
    const int q = rr * CPR + lane / L;
    const int w0 = lane % L;
    V v = V(0);
    if (q < NC) {
#pragma unroll
      for (int j = 0; j < PER; ++j) v += base[(w0 + j * L) * stride + q];
    }
#pragma unroll
    for (int off = L / 2; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
#pragma unroll
    for (int c = 0; c < CPR; ++c)
      if (rr * CPR + c < NC) tot[rr * CPR + c] = __shfl_sync(0xffffffffu, v, c * L);
  }
}


// Set-up variant of fused_block: the axpy uses coef = α_j; the next group's statistics are
// per-vector FP32 partial sums of <= 8 values (BF16 squares are exact in FP32) folded into
// FP64 accumulators (Σa, Σa²).
template <typename Elem, int R, int GC, bool NEXT, int TC>
__device__ __forceinline__ void fused_block_setup(const unsigned char* cur, const unsigned char* nxt,
                                                  uint32_t col_bytes, int t, int T_rt,
                                                  const float (&coef)[GC],
                                                  float2 (&yacc)[R][8 / sizeof(Elem)],
                                                  double2 (&dn)[GC]) {
  constexpr int H = 8 / sizeof(Elem);
  const int T = TC > 0 ? TC : T_rt;
  const int colv = TC > 0 ? R * TC : (int)(col_bytes >> 4);
  const uint4* c4 = reinterpret_cast<const uint4*>(cur) + t;
  const uint4* n4 = reinterpret_cast<const uint4*>(nxt) + t;
  // FP32 partial sums over this thread's R vectors of a column (the BF16 squares are exact in
  // FP32), folded into FP64 once per column
  float2 s2[GC], q2[GC];
#pragma unroll
  for (int qq = 0; qq < GC; ++qq) {
    s2[qq] = make_float2(0.f, 0.f);
    q2[qq] = make_float2(0.f, 0.f);
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    uint4 vc[GC], vn[GC];
#pragma unroll
    for (int qq = 0; qq < GC; ++qq) {
      vc[qq] = c4[qq * colv + r * T];
      if (NEXT) vn[qq] = n4[qq * colv + r * T];
    }
#pragma unroll
    for (int qq = 0; qq < GC; ++qq) {
      float2 ac[H];
      unpack2(vc[qq], ac);
      const float2 c2 = make_float2(coef[qq], coef[qq]);
#pragma unroll
      for (int h = 0; h < H; ++h) yacc[r][h] = fma2(c2, ac[h], yacc[r][h]);
      if (NEXT) {
        float2 an[H];
        unpack2(vn[qq], an);
#pragma unroll
        for (int h = 0; h < H; ++h) {
          s2[qq] = __fadd2_rn(s2[qq], an[h]);
          q2[qq] = fma2(an[h], an[h], q2[qq]);
        }
      }
    }
  }
#pragma unroll
  for (int qq = 0; qq < GC; ++qq)
    dn[qq] = make_double2((double)s2[qq].x + (double)s2[qq].y,
                          (double)q2[qq].x + (double)q2[qq].y);
}

template <typename Elem, int R, int GC, bool SETUP>
__global__ void __launch_bounds__(kMaxThreads, 1)
    panel_kernel(const __grid_constant__ PanelArgs a) {
  using RT = typename RedT<SETUP>::T;
  constexpr int E = 16 / static_cast<int>(sizeof(Elem));
  constexpr int H = E / 2;  // float2 per vector
  const Buffers& b = a.b;
  const PanelGeom& g = a.g;
  const CallCfg& cc = a.cc;
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const int T = blockDim.x;  // threads: all consume; thread 0 also issues the copies
  const int ncw = T >> 5;    // warps
  const int G = gridDim.x;
  const int q = blockIdx.x;
  const int m = b.m;
  const double inv_m = 1.0 / (double)m;
  const int nvec = m / E;
  const int NS = g.nstages;
  const uint32_t col_bytes = (uint32_t)(m * sizeof(Elem));
  const bool full_slots = (T * R == nvec);  // every vector slot of every thread is a real row

  extern __shared__ __align__(128) unsigned char smem[];
  const SmemLayout L = smem_layout(g, SETUP);
  unsigned char* stages = smem + L.stages;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + L.bars);
  RT* redw = reinterpret_cast<RT*>(smem + L.redw);
  uint32_t* wl_idx = reinterpret_cast<uint32_t*>(smem + L.wl_idx);
  float* wl_w = reinterpret_cast<float*>(smem + L.wl_w);
  float* wl_al = reinterpret_cast<float*>(smem + L.wl_al);
  uint32_t* nxt_cols = reinterpret_cast<uint32_t*>(smem + L.nxt);  // [kGcMax * 8]
  double4* red = reinterpret_cast<double4*>(smem + L.red);          // [16 warps][32]
  float4* epi_yp = reinterpret_cast<float4*>(smem + L.epi);          // [32] each
  float4* epi_ym = epi_yp + 32;
  float4* epi_v = epi_yp + 64;
  float4* epi_xm = epi_yp + 96;
  float4* epi_z = epi_yp + 128;
  double* epi_vs = reinterpret_cast<double*>(epi_yp + 160);          // [32][4]
  __shared__ IterState st_s;   // state of the current step, identical in every CTA
  __shared__ int32_t pre_s[2];  // groups of the current step issued ahead, and their list key
  __shared__ uint32_t cd_s[kListWindow];  // work-list lengths of the slots (fixed per launch)
  __shared__ int32_t nx_s[4];   // predicted next list: groups to issue ahead, key, length, sampled
  __shared__ int64_t nxlo_s;    // ... and its first index
  __shared__ uint32_t iss_s;    // groups issued so far (thread 0)
  __shared__ IterState nxs_s;   // the next state, formed by warp 0
  __shared__ int32_t wlkey_s;   // slot of the coefficient slice copied ahead into wl_* (-2: none)
  __shared__ uint32_t xstage_s; // clusters: the stage holding this CTA's partial y (read by peers)

  // A launch of the step kernel is a programmatic dependent of the grid before it: its CTAs
  // start on the SMs that the previous grid leaves, initialise their barriers, and wait for
  // that grid to complete before touching global memory.  Every CTA of this grid is resident
  // by the time it lets the next grid be scheduled (one CTA per SM), so the grid barriers
  // below are unaffected.
  if (!SETUP) griddep_launch_dependents();
  // Clusters (CL > 1): the partial-y exchange of each step runs on two mbarriers per CTA, each
  // completing when all CL CTAs of the cluster have arrived (remote arrives): xbar[0] when every
  // CTA has published its partial in shared memory, xbar[1] when every CTA is done reading its
  // peers'.  A CTA refills the stage holding its partial, or leaves the kernel, only after
  // xbar[1] of its last exchange (bounded waits throughout: no hardware cluster barrier after
  // the prologue, so no CTA can be held by a peer that gave up).
  const int CL = g.cluster;
  uint64_t* xbar = full + 8;
  if (t == 0) {
    for (int s = 0; s < NS; ++s) mbar_init(&full[s], 1);
    if (CL > 1) {
      mbar_init(&xbar[0], (uint32_t)CL);
      mbar_init(&xbar[1], (uint32_t)CL);
    }
    fence_barrier_init();
  }
  __syncthreads();  // barrier initialisation visible to every thread
  // every CTA of the cluster has initialised its barriers before any peer arrives on them (no
  // CTA can have left the kernel yet)
  if (CL > 1) cluster_sync_all();
  if (!SETUP) griddep_wait();

  // work-list lengths of every slot (fixed for the launch: the window is refilled between
  // launches) and the state of the launch's first step; loop-carried values live in shared
  // memory, so that the group loop keeps its registers
  if (!SETUP) {
    if (t < kListWindow) cd_s[t] = __ldg(b.wl_count + t);
    if (t == 0) {
      st_s = b.st[a.iter & 1];
      pre_s[0] = 0;
      pre_s[1] = -2;
      wlkey_s = -2;
    }
  }
  if (t == 0) iss_s = 0u;
  // this CTA's rows of the grid-wide epilogue: float4 row groups [g0, g1)
  const int RG = m >> 2;
  const int g0 = (int)((int64_t)q * RG / G), g1 = (int)((int64_t)(q + 1) * RG / G);
  // The first 32 of them are kept in shared memory for the whole launch: y_{i-1}, y_memo,
  // x_memo (the epilogue rewrites them as it produces y_i and a new memo pair), v, z and v*.
  if (!SETUP && warp == (ncw > 2 ? 2 : 0) && g0 + lane < g1) {
    const int row = 4 * (g0 + lane);
    epi_yp[lane] = __ldcg(reinterpret_cast<const float4*>(b.y[(a.iter + 1) & 1] + row));
    epi_ym[lane] = __ldcg(reinterpret_cast<const float4*>(b.y_memo + row));
    epi_xm[lane] = __ldcg(reinterpret_cast<const float4*>(b.x_memo + row));
    epi_v[lane] = __ldcg(reinterpret_cast<const float4*>(b.v + row));
    epi_z[lane] = __ldcg(reinterpret_cast<const float4*>(b.z + row));
#pragma unroll
    for (int e = 0; e < 4; ++e) epi_vs[lane * 4 + e] = b.has_vstar ? __ldcg(b.vstar + row + e) : 0.0;
  }
  // this thread's rows of y_{j-1} (and of x_memo when it is not known to be zero) for step j
  float4 ypv[R][E / 4], xmv[R][E / 4];
  auto load_vecs = [&](int j, bool memo) {
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int vi = t + r * T;
#pragma unroll
      for (int h4 = 0; h4 < E / 4; ++h4) {
        ypv[r][h4] = make_float4(0.f, 0.f, 0.f, 0.f);
        xmv[r][h4] = ypv[r][h4];
        if (!SETUP && vi < nvec) {
          const int o4 = vi * (E / 4) + h4;
          ypv[r][h4] = __ldcg(reinterpret_cast<const float4*>(b.y[(j + 1) & 1]) + o4);
          if (memo) xmv[r][h4] = __ldcg(reinterpret_cast<const float4*>(b.x_memo) + o4);
        }
      }
    }
  };


  // this CTA's slice [lo, hi) of the column list of a step reading `cd` sampled columns
  // (sampled) or all n columns
  auto slice = [&](bool smp, uint32_t cd, int64_t& lo, int64_t& hi) {
    const int64_t total = smp ? (int64_t)cd : (int64_t)b.n;
    lo = (int64_t)q * total / G;
    hi = (int64_t)(q + 1) * total / G;
  };

  // Stage ring: group number `pos` (counted over the whole launch) lives in stage pos % NS and
  // completes phase (pos / NS) of that stage's barrier.  Thread 0 issues; a stage is refilled
  // once every thread is past the group that last used it (the CTA barrier ending each group).
  const uint64_t policy = l2_evict_first_policy();
  const size_t col_stride = (size_t)b.ld * sizeof(Elem);
  const unsigned char* Abase = reinterpret_cast<const unsigned char*>(b.A);
  auto issue_at = [&](uint32_t pos, int cnt, const uint32_t* cols, int64_t first_col) {
    const int s = (int)(pos % (uint32_t)NS);
    mbar_arrive_expect_tx(&full[s], (uint32_t)cnt * col_bytes);
    for (int qq = 0; qq < cnt; ++qq) {
      const uint32_t col = cols ? cols[qq] : (uint32_t)(first_col + qq);
      bulk_g2s(stages + ((size_t)s * GC + qq) * col_bytes, Abase + (size_t)col * col_stride,
               col_bytes, &full[s], policy);
    }
  };
  auto wait_pos = [&](uint32_t pos) -> bool {
    return mbar_wait_bounded(&full[pos % (uint32_t)NS], (pos / (uint32_t)NS) & 1u);
  };
  uint32_t gbase = 0;   // groups through the ring before the current step (every thread)
  bool ok = true;
  // on the way out: no copy may still be landing in this CTA's shared memory (the last NS
  // issued groups cover every stage; waits are bounded)
  auto drain = [&]() {
    if (t == 0) {
      const uint32_t issued = iss_s;
      for (uint32_t p = issued > (uint32_t)NS ? issued - (uint32_t)NS : 0u; p < issued; ++p)
        wait_pos(p);
    }
  };
  // partial-y exchanges of the cluster completed by this CTA (uniform over its threads)
  uint32_t npub = 0;
  auto xarrive = [&](int which) {  // thread r < CL arrives on rank r's barrier
    if (t < CL) mbar_arrive_remote(map_to_rank(smem_addr(&xbar[which]), (uint32_t)t));
  };
  // before leaving the kernel: the peers are done with this CTA's shared memory
  auto xsettle = [&]() {
    if (CL > 1 && npub > 0) mbar_wait_cluster_bounded(&xbar[1], (npub - 1) & 1u);
  };
  // this step's exchange without data, on a failure path: the peers waiting on this CTA are
  // released, and it leaves only once they are done with its shared memory
  auto xabandon = [&]() {
    if (CL <= 1) return;
    named_barrier_or(1, T, false);
    xarrive(0);
    mbar_wait_cluster_bounded(&xbar[0], npub & 1u);
    named_barrier_or(1, T, false);
    xarrive(1);
    ++npub;
    xsettle();
  };

  // ---- everything step j needs that does not depend on the product of the step before ----
  // dx = x_j − x_memo on this thread's rows (x_j = scale·y_{j−1}, FP32 multiply) and the CTA's
  // Σdx; one warp's z·dx over this CTA's rows (dots, common.h:55-87, into rpart[4q+3]) and the
  // epilogue's inputs of its first 32 row groups; the coefficient slice of the step's list; and
  // the list predicted for step j+1 (exact unless the adaptive VR switch, which needs step j's
  // cosine, changes the kind), whose first column indices thread 0 issues as soon as step j's
  // last group is consumed, so that HBM stays busy through the grid-wide epilogue.  Run for the
  // first step of the launch, and for each later step right after the state is formed.
  float2 dx[R][H];
  double sum_dx = 0.0;
  auto prepare = [&](int j, const IterState& sj) {
    const bool jamm = sj.mode == kPrevious || sj.mode == kProposed;
    const bool jcentred = sj.mode == kProposed;
    const bool jsampled = jamm && !cc.sanity;
    const int jslot = sj.used % kListWindow;
    const float jscale = sj.scale;
    int64_t jlo, jhi;
    slice(jsampled, cd_s[jslot], jlo, jhi);
    const int jnb = (int)(jhi - jlo);
    const float* yprev = b.y[(j + 1) & 1];
    load_vecs(j, jamm && !sj.memo_zero);
    if (warp == (ncw > 2 ? 2 : 0)) {
      if (jcentred) {
        double zp = 0.0;
        for (int c0 = g0; c0 < g1; c0 += 32) {
          const int gi = c0 + lane;
          if (gi < g1) {
            const int row = 4 * gi;
            const bool st0 = c0 == g0;  // the first 32 row groups are in shared memory
            const float4 yp = st0 ? epi_yp[lane] : __ldcg(reinterpret_cast<const float4*>(yprev + row));
            const float4 xm = st0 ? epi_xm[lane] : __ldcg(reinterpret_cast<const float4*>(b.x_memo + row));
            const float4 z4 = st0 ? epi_z[lane] : __ldcg(reinterpret_cast<const float4*>(b.z + row));
            zp = fma((double)__fsub_rn(__fmul_rn(jscale, yp.x), xm.x), (double)z4.x, zp);
            zp = fma((double)__fsub_rn(__fmul_rn(jscale, yp.y), xm.y), (double)z4.y, zp);
            zp = fma((double)__fsub_rn(__fmul_rn(jscale, yp.z), xm.z), (double)z4.z, zp);
            zp = fma((double)__fsub_rn(__fmul_rn(jscale, yp.w), xm.w), (double)z4.w, zp);
          }
        }
        zp = warp_sum(zp);
        if (lane == 0) b.rpart[4 * q + 3] = zp;
      }
    }
    // the coefficient slice, unless copied ahead on the right prediction (the warps after warp
    // 0, all of a one-warp CTA)
    if (jamm && !(jsampled && wlkey_s == jslot)) {
      cp_async_wait_all();  // no copy ahead may still land in wl_*
      const int t1 = T > 32 ? t - 32 : t, T1 = T > 32 ? T - 32 : T;
      for (int k = t1; k >= 0 && k < jnb; k += T1) {
        if (jsampled) {
          wl_idx[k] = __ldg(b.wl_col[jslot] + jlo + k);
          wl_w[k] = __ldg(b.wl_wm[jslot] + jlo + k);
          wl_al[k] = __ldg(b.wl_al[jslot] + jlo + k);
        } else {  // sanity mode: identity list, weight 1
          wl_w[k] = 1.0f;
          wl_al[k] = __ldg(b.alpha + jlo + k);
        }
      }
    }
    if (warp == (ncw > 1 ? 1 : 0)) {
      int groups = 0, nkey = -2, nnb = 0, nsmp = 0;
      int64_t nlo = 0;
      if (j + 1 < a.iter_end) {
        int le;
        const int nmode = decide_mode(cc, j + 1, sj.cos_prev, sj.last_exact, &le);
        const int nslot = (sj.used + (jsampled ? 1 : 0)) % kListWindow;
        nsmp = ((nmode == kPrevious || nmode == kProposed) && !cc.sanity) ? 1 : 0;
        int64_t nhi;
        slice(nsmp != 0, cd_s[nslot], nlo, nhi);
        nnb = (int)(nhi - nlo);
        groups = min(NS, (nnb + GC - 1) / GC);
        nkey = nsmp ? nslot : -1;
        if (nsmp) {
          const int nf = min(NS * GC, nnb);
          for (int k = lane; k < nf; k += 32) cp_async4(nxt_cols + k, b.wl_col[nslot] + nlo + k);
        }
      }
      if (lane == 0) {
        nx_s[0] = groups;
        nx_s[1] = nkey;
        nx_s[2] = nnb;
        nx_s[3] = nsmp;
        nxlo_s = nlo;
      }
    }
    double sdx = 0.0;
#pragma unroll
    for (int r = 0; r < R; ++r) {
#pragma unroll
      for (int h4 = 0; h4 < E / 4; ++h4) {
        const float4 yp = ypv[r][h4];
        const float4 xm = jamm ? xmv[r][h4] : make_float4(0.f, 0.f, 0.f, 0.f);
        const float d0 = __fsub_rn(__fmul_rn(jscale, yp.x), xm.x);
        const float d1 = __fsub_rn(__fmul_rn(jscale, yp.y), xm.y);
        const float d2 = __fsub_rn(__fmul_rn(jscale, yp.z), xm.z);
        const float d3 = __fsub_rn(__fmul_rn(jscale, yp.w), xm.w);
        dx[r][2 * h4] = make_float2(d0, d1);
        dx[r][2 * h4 + 1] = make_float2(d2, d3);
        if (jcentred) sdx += ((double)d0 + (double)d1) + ((double)d2 + (double)d3);
      }
    }
    sum_dx = 0.0;
    if (jcentred) {  // Σdx over all m rows (dots, common.h:55-87), identical in every CTA
      sdx = warp_sum(sdx);
      double* wtmp = reinterpret_cast<double*>(redw);
      if (lane == 0) wtmp[warp] = sdx;
      named_barrier_or(1, T, false);
      for (int w = 0; w < ncw; ++w) sum_dx += wtmp[w];
      named_barrier_or(1, T, false);  // wtmp (= redw) is reused by the group loop
    }
  };
  if (!SETUP) {
    __syncthreads();  // st_s
    if (a.iter < a.iter_end && !st_s.done) prepare(a.iter, st_s);  // uniform over the grid
  }

  for (int i = a.iter;; ++i) {
    int mode = kExact, slot = 0;
    float scale = 0.f;
    if (!SETUP) {
      __syncthreads();  // st_s and pre_s of this step; every thread is done with the last one
      if (i >= a.iter_end || st_s.done) break;  // uniform over the grid
      mode = st_s.mode;
      slot = st_s.used % kListWindow;
      scale = st_s.scale;
    }
    const bool amm = !SETUP && (mode == kPrevious || mode == kProposed);
    const bool centred = !SETUP && mode == kProposed;
    const bool sampled = amm && !cc.sanity;
    const int key = sampled ? slot : -1;  // which columns the step reads

    // ---- this CTA's column list: a contiguous slice of the sorted work list ----------------
    const uint32_t cd = SETUP ? 0u : cd_s[slot];
    int64_t lo, hi;
    slice(sampled, cd, lo, hi);
    if (sampled && q == 0 && t == 0) b.distinct_hist[i] = (int32_t)cd;
    const int nb = (int)(hi - lo);
    const int ngroups = (nb + GC - 1) / GC;
    const uint32_t* list_col = sampled ? b.wl_col[slot] + lo : nullptr;

    // the groups of this step already in flight (issued at the end of the previous step on
    // the predicted list); a misprediction is drained and the ring position moves past it
    int pre = 0;
    if (!SETUP) {
      const int pn = pre_s[0];
      if (pn > 0) {
        if (pre_s[1] == key) {
          pre = pn;
        } else {
          if (t == 0)
            for (int k = 0; k < pn; ++k) wait_pos(gbase + (uint32_t)k);
          gbase += (uint32_t)pn;
        }
      }
    }

    // the stage that held this CTA's partial of the last exchange is refilled below: the
    // peers must be done reading it (already so in practice: two grid barriers lie between)
    if (CL > 1 && npub > 0 && t == 0) {
      if (!mbar_wait_cluster_bounded(&xbar[1], (npub - 1) & 1u)) ok = false;
      fence_proxy_async_smem();  // generic writes of the partial before the async refill
    }
    if (t == 0 && ok && ngroups > pre) {  // the first NS groups not already in flight
      uint32_t first[kGcMax * 8];
      const int nf = min(NS * GC, nb);
      if (sampled)
        for (int k = pre * GC; k < nf; ++k) first[k] = __ldg(list_col + k);
      for (int grp = pre; grp < NS && grp < ngroups; ++grp)
        issue_at(gbase + (uint32_t)grp, min(GC, nb - grp * GC), sampled ? first + grp * GC : nullptr,
                 lo + grp * GC);
      iss_s = gbase + (uint32_t)min(NS, ngroups);
    }

    float2 yacc[R][H];
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int h = 0; h < H; ++h) yacc[r][h] = make_float2(0.f, 0.f);
    double zdx = 0.0;
    const float sum_dx_f = (float)sum_dx;

    // ring slot (stage, phase parity) of group 0 of this step; the group loop advances it
    const uint32_t stage_bytes = (uint32_t)GC * col_bytes;
    int s_cur = (int)(gbase % (uint32_t)NS);
    uint32_t ph_cur = (gbase / (uint32_t)NS) & 1u;
    // guarded partial dots of the group in stage s (tail groups, partial slots, the set-up
    // statistics)
    auto dot_group = [&](int grp, int s, RT (&d)[GC], bool got) -> bool {
      const int cnt = got ? min(GC, nb - grp * GC) : 0;
      const unsigned char* sb = stages + (size_t)s * stage_bytes;
#pragma unroll
      for (int qq = 0; qq < GC; ++qq) {
        if constexpr (SETUP) {
          d[qq] = make_double2(0.0, 0.0);
        } else {
          d[qq] = 0.f;
        }
        if (qq < cnt) {
          const uint4* col = reinterpret_cast<const uint4*>(sb + (size_t)qq * col_bytes);
          if constexpr (SETUP) {
            // FP32 partial sums over this thread's vectors, folded into FP64 once (as
            // fused_block_setup)
            float2 s2 = make_float2(0.f, 0.f), q2 = make_float2(0.f, 0.f);
#pragma unroll
            for (int r = 0; r < R; ++r) {
              const int vi = t + r * T;
              if (vi < nvec) {
                float2 av[H];
                unpack2(col[vi], av);
#pragma unroll
                for (int h = 0; h < H; ++h) {
                  s2 = __fadd2_rn(s2, av[h]);
                  q2 = fma2(av[h], av[h], q2);
                }
              }
            }
            d[qq] = make_double2((double)s2.x + (double)s2.y, (double)q2.x + (double)q2.y);
          } else {
            float2 p0 = make_float2(0.f, 0.f), p1 = make_float2(0.f, 0.f);
#pragma unroll
            for (int r = 0; r < R; ++r) {
              const int vi = t + r * T;
              if (vi < nvec) {
                float2 av[H];
                unpack2(col[vi], av);
#pragma unroll
                for (int h = 0; h < H; h += 2) {
                  p0 = fma2(av[h], dx[r][h], p0);
                  if (h + 1 < H) p1 = fma2(av[h + 1], dx[r][h + 1], p1);
                }
              }
            }
            d[qq] = (p0.x + p0.y) + (p1.x + p1.y);
          }
        }
      }
      return got;
    };
    auto publish = [&](int grp, RT (&d)[GC]) {
      const int cnt = min(GC, nb - grp * GC);
      RT* slotp = redw + ((grp & 1) * 16 + warp) * GC;
      if constexpr (!SETUP && GC >= 2) {
        float v[GC];
#pragma unroll
        for (int qq = 0; qq < GC; ++qq) v[qq] = d[qq];
        const float r = warp_reduce_multi<float, GC>(v, lane);
        constexpr int LL = 32 / GC;
        const int qv = lane / LL;
        if (lane % LL == 0 && qv < cnt) slotp[qv] = r;
      } else if constexpr (SETUP && 2 * GC <= 32) {
        double v[2 * GC];
#pragma unroll
        for (int qq = 0; qq < GC; ++qq) {
          v[2 * qq] = d[qq].x;
          v[2 * qq + 1] = d[qq].y;
        }
        const double r = warp_reduce_multi<double, 2 * GC>(v, lane);
        constexpr int LL = 32 / (2 * GC);
        const int idx = lane / LL;
        if (lane % LL == 0 && (idx >> 1) < cnt) {
          double* sd = reinterpret_cast<double*>(slotp);
          sd[idx] = r;  // (Σa, Σa²) of column idx/2
        }
      } else {
#pragma unroll
        for (int qq = 0; qq < GC; ++qq) {
          if (qq < cnt) {
            const RT v = warp_red(d[qq]);
            if (lane == 0) slotp[qq] = v;
          }
        }
      }
    };

    float sacc = 0.f;    // Σ α_k t_k (proposed)
    double a2acc = 0.0;  // Σ α_j² (set-up)
    RT dn[GC];
    if (ngroups > 0) {
      ok = mbar_wait_bounded(&full[s_cur], ph_cur);
      dot_group(0, s_cur, dn, ok);
      publish(0, dn);
    }
    cp_async_wait_all();  // the slice and next-list indices copied ahead, published below
    if (named_barrier_or(1, T, !ok)) ok = false;
    for (int grp = 0; ok && grp < ngroups; ++grp) {
      const int cnt = min(GC, nb - grp * GC);
      // coefficients of this group (every thread sums the warp partials in the same order)
      float coef[GC];
      const RT* rs = redw + (grp & 1) * 16 * GC;
      float tots[GC];
      double sxy[2 * GC];
      if constexpr (SETUP) {
        const double* rsd = reinterpret_cast<const double*>(rs);
        if (ncw == 16) {
          warp_partials_sum<double, 2 * GC>(rsd, 2 * GC, lane, sxy);
        } else {
#pragma unroll
          for (int k = 0; k < 2 * GC; ++k) {
            double tt = rsd[k];
            for (int w = 1; w < ncw; ++w) tt += rsd[w * 2 * GC + k];
            sxy[k] = tt;
          }
        }
      } else {
        if (ncw == 16) {
          warp_partials_sum<float, GC>(reinterpret_cast<const float*>(rs), GC, lane, tots);
        } else {
#pragma unroll
          for (int qq = 0; qq < GC; ++qq) {
            float tt = rs[qq];
            for (int w = 1; w < ncw; ++w) tt += rs[w * GC + qq];
            tots[qq] = tt;
          }
        }
      }
#pragma unroll
      for (int qq = 0; qq < GC; ++qq) {
        coef[qq] = 0.f;
        if (qq < cnt) {
          const int k = grp * GC + qq;
          if constexpr (SETUP) {
            // α_j = Σa·(1/m) (exactly Σa/m for a power-of-two m); the sums go to colsum and
            // the column statistics are formed in the epilogue, off this per-group path
            const double sx = sxy[2 * qq];
            const float af = (float)(sx * inv_m);
            coef[qq] = af;
            a2acc = fma((double)af, (double)af, a2acc);
            if (t == qq) b.colsum[lo + k] = make_double2(sx, sxy[2 * qq + 1]);
          } else {
            const float tot = tots[qq];
            if (!amm) {
              coef[qq] = tot;
            } else if (centred) {
              const float al = wl_al[k];
              const float tq = __fmul_rn(__fsub_rn(tot, __fmul_rn(al, sum_dx_f)), wl_w[k]);
              coef[qq] = tq;
              sacc = fmaf(al, tq, sacc);
            } else {
              coef[qq] = __fmul_rn(tot, wl_w[k]);
            }
          }
        }
      }
      const bool more = grp + 1 < ngroups;
      const int cnt_n = more ? min(GC, nb - (grp + 1) * GC) : 0;
      const int s_nxt = s_cur + 1 == NS ? 0 : s_cur + 1;
      const uint32_t ph_nxt = s_nxt == 0 ? ph_cur ^ 1u : ph_cur;
      bool got = true;
      if (more) got = mbar_wait_bounded(&full[s_nxt], ph_nxt);
      ok = ok && got;
      const unsigned char* sb = stages + (size_t)s_cur * stage_bytes;
      bool fused = false;
      if (full_slots && cnt == GC && got) {
        const unsigned char* sn = more ? stages + (size_t)s_nxt * stage_bytes : sb;
        if constexpr (SETUP) {
          if (more && cnt_n == GC) {
            if (T == 512)
              fused_block_setup<Elem, R, GC, true, 512>(sb, sn, col_bytes, t, T, coef, yacc, dn);
            else
              fused_block_setup<Elem, R, GC, true, 0>(sb, sn, col_bytes, t, T, coef, yacc, dn);
            fused = true;
          } else if (!more) {
            if (T == 512)
              fused_block_setup<Elem, R, GC, false, 512>(sb, sb, col_bytes, t, T, coef, yacc, dn);
            else
              fused_block_setup<Elem, R, GC, false, 0>(sb, sb, col_bytes, t, T, coef, yacc, dn);
            fused = true;
          }
        } else {
          if (more && cnt_n == GC) {
            if (T == 512)
              fused_block<Elem, R, GC, true, 512>(sb, sn, col_bytes, t, T, coef, dx, yacc, dn);
            else
              fused_block<Elem, R, GC, true, 0>(sb, sn, col_bytes, t, T, coef, dx, yacc, dn);
            fused = true;
          } else if (!more) {
            if (T == 512)
              fused_block<Elem, R, GC, false, 512>(sb, sb, col_bytes, t, T, coef, dx, yacc, dn);
            else
              fused_block<Elem, R, GC, false, 0>(sb, sb, col_bytes, t, T, coef, dx, yacc, dn);
            fused = true;
          }
        }
      }
      if (!fused) {
        // partial dots of the next group (its reduction latency overlaps this group's axpy)
        if (more) dot_group(grp + 1, s_nxt, dn, got);
        // y += coef · A over this thread's rows
#pragma unroll
        for (int qq = 0; qq < GC; ++qq) {
          if (qq < cnt) {
            const uint4* col = reinterpret_cast<const uint4*>(sb + (size_t)qq * col_bytes);
            const float2 c2 = make_float2(coef[qq], coef[qq]);
#pragma unroll
            for (int r = 0; r < R; ++r) {
              const int vi = t + r * T;
              if (vi < nvec) {
                float2 av[H];
                unpack2(col[vi], av);
#pragma unroll
                for (int h = 0; h < H; ++h) yacc[r][h] = fma2(c2, av[h], yacc[r][h]);
              }
            }
          }
        }
      }
      if (more) publish(grp + 1, dn);
      // partials of grp+1 published; every thread is done with stage grp: thread 0 refills it
      if (named_barrier_or(1, T, !ok)) ok = false;
      if (t == 0 && ok && grp + NS < ngroups) {
        // group grp + NS takes the stage of group grp
        const int c0 = (grp + NS) * GC;
        const int cn = min(GC, nb - c0);
        mbar_arrive_expect_tx(&full[s_cur], (uint32_t)cn * col_bytes);
        for (int qq = 0; qq < cn; ++qq) {
          const uint32_t col = sampled ? wl_idx[c0 + qq] : (uint32_t)(lo + c0 + qq);
          bulk_g2s(stages + (size_t)s_cur * stage_bytes + (size_t)qq * col_bytes,
                   Abase + (size_t)col * col_stride, col_bytes, &full[s_cur], policy);
        }
        iss_s = gbase + (uint32_t)(grp + NS + 1);
      }
      s_cur = s_nxt;
      ph_cur = ph_nxt;
    }
    if (!ok) {
      xabandon();
      drain();
      if (t == 0) atomicOr(b.status, (uint32_t)kDevTimeout);
      return;
    }
    gbase += (uint32_t)ngroups;
    // every stage is free: the next step's first groups go out now (thread 0).  Two groups
    // (about 128 KB per CTA): measured on the B200, a third one slows the partial-sum writes
    // and the grid barrier that follow by more than it saves, and issuing them after the
    // barrier arrival gains nothing.
    if (!SETUP && t == 0) {
      const int groups = min(nx_s[0], kPrefetchGroups), nnb = nx_s[2];
      const bool nsmp = nx_s[3] != 0;
      const int64_t nlo = nxlo_s;
      for (int grp = 0; grp < groups; ++grp)
        issue_at(gbase + (uint32_t)grp, min(GC, nnb - grp * GC),
                 nsmp ? nxt_cols + grp * GC : nullptr, nlo + grp * GC);
      if (groups > 0) iss_s = gbase + (uint32_t)groups;
      pre_s[0] = groups;
      pre_s[1] = nx_s[1];
    }

    if (sampled) {
      // The picks are consumed: their histogram entries and chunk totals are cleared for the
      // next draw into this slot (several CTAs may zero one chunk total: the same value).
      const int cs = b.chunk_shift;
      uint32_t* cnt = b.count[slot];
      uint32_t* chk = b.chunk[slot];
      for (int k = t; k < nb; k += T) {
        const uint32_t col = wl_idx[k];  // written before the barriers of the group loop
        cnt[col] = 0u;
        chk[col >> cs] = 0u;
      }
    }
    // this CTA's partial y: to the partial-sum buffer, or (clusters) to a stage that no copy
    // uses (at most kPrefetchGroups of the NS >= 3 stages hold the next step's first groups;
    // which one depends on this CTA's ring position, so it is published for the peers)
    const uint32_t xstage = (gbase + kPrefetchGroups) % (uint32_t)NS;
    if (CL > 1 && t == 0) xstage_s = xstage;
    float* part = CL > 1 ? reinterpret_cast<float*>(stages + (size_t)xstage * stage_bytes)
                         : b.partials + (size_t)q * m;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int vi = t + r * T;
      if (vi < nvec) {
#pragma unroll
        for (int h4 = 0; h4 < E / 4; ++h4)
          reinterpret_cast<float4*>(part)[vi * (E / 4) + h4] =
              make_float4(yacc[r][2 * h4].x, yacc[r][2 * h4].y, yacc[r][2 * h4 + 1].x,
                          yacc[r][2 * h4 + 1].y);
      }
    }
    if (t == 0) {
      b.spart[q] = sacc;
      b.spart64[q] = a2acc;
    }
    if (CL > 1) {
      // The cluster's partial: CTA rank r sums float4 row groups [r·m/(4·CL), (r+1)·m/(4·CL))
      // of the CL partials in rank order (FP32) from the peers' shared memory, and writes them
      // to the cluster's partial-sum row.
      fence_acq_rel_cluster();
      named_barrier_or(1, T, false);  // the whole partial is in shared memory
      xarrive(0);
      const bool got = mbar_wait_cluster_bounded(&xbar[0], npub & 1u);
      const bool bad = named_barrier_or(1, T, !got);
      if (!bad) {
        const int per = (m >> 2) / CL;
        const int r0 = (int)cluster_ctarank() * per;
        // each peer's partial: its stage index, then the stage's address in its shared memory
        uint32_t fa[8];
        const uint32_t sbase = smem_addr(stages), xs_addr = smem_addr(&xstage_s);
        for (int k = 0; k < CL; ++k) {
          uint32_t ks;
          asm volatile("ld.shared::cluster.u32 %0, [%1];"
                       : "=r"(ks)
                       : "r"(map_to_rank(xs_addr, (uint32_t)k))
                       : "memory");
          fa[k] = map_to_rank(sbase + ks * stage_bytes, (uint32_t)k);
        }
        float4* cpart = reinterpret_cast<float4*>(b.partials + (size_t)(q / CL) * m);
        for (int gi = r0 + t; gi < r0 + per; gi += T) {
          float4 acc = ld_cluster_f4(fa[0] + 16u * (uint32_t)gi);
          for (int k = 1; k < CL; ++k) {
            const float4 v = ld_cluster_f4(fa[k] + 16u * (uint32_t)gi);
            acc.x += v.x;
            acc.y += v.y;
            acc.z += v.z;
            acc.w += v.w;
          }
          cpart[gi] = acc;
        }
      }
      named_barrier_or(1, T, false);  // this CTA is done reading its peers
      xarrive(1);
      ++npub;
      if (bad) {
        xsettle();
        drain();
        if (t == 0) atomicOr(b.status, (uint32_t)kDevTimeout);
        return;
      }
    }

    // ====================== the step's epilogue, fused (grid-wide) ======================
    // Every CTA is resident (one per SM), so after a grid barrier the G partials are summed
    // where they sit in L2: CTA q owns float4 row groups [g0, g1) and sums them over the CTAs
    // in a fixed order (FP64); then the new y rows and this CTA's share of the Rayleigh sums
    // (dotProduct_and_generate_x, common.h:103-153); after a second grid barrier every CTA
    // forms λ and the next step's state from the CTA shares, in the same order.
    const float* yprev = b.y[(i + 1) & 1];
    float* ynew = b.y[i & 1];
    named_barrier_or(1, T, false);  // this CTA's partials are written
    bool bar_ok = true;
    if (t == 0) bar_ok = grid_barrier(b.ticket + 2, (uint32_t)G);
    if (named_barrier_or(1, T, !bar_ok)) {
      xsettle();
      drain();
      if (t == 0) atomicOr(b.status, (uint32_t)kDevTimeout);
      return;
    }
    double S = 0.0;  // Σ over the CTAs of the per-CTA scalar (fixed order, the same everywhere)
    double xy = 0.0, yy = 0.0, yv = 0.0;
    const int NPART = G / CL;  // partial-sum rows: one per CTA, or one per cluster
    constexpr int kU = 10;
    // The per-CTA scalars (Σ α_k t_k and z·dx of the proposed step, Σ α_j² of the set-up pass)
    // reach shared memory with one load per thread, issued together with the partial-sum loads
    // (one L2 round trip); warp 0 then sums them from shared memory in a fixed order.
    const bool want_s = SETUP || centred;
    double* scal = reinterpret_cast<double*>(smem + L.scal);
    auto sval = [&](int k) -> double {  // entry k of [per-CTA scalar | z·dx]
      if constexpr (SETUP) {
        return k < G ? __ldcg(b.spart64 + k) : 0.0;
      } else {
        return k < G ? (double)__ldcg(b.spart + k) : __ldcg(b.rpart + 4 * (k - G) + 3);
      }
    };
    for (int c0 = g0; c0 < g1; c0 += 32) {
      const int gi = c0 + lane;
      const bool first = (c0 == g0);
      double4 acc = make_double4(0.0, 0.0, 0.0, 0.0);
      const bool sload = first && want_s && t < 2 * G;
      const double sreg = sload ? sval(t) : 0.0;
      if (gi < g1) {
        const float* P = b.partials + 4 * (size_t)gi;
        for (int k0 = warp; k0 < NPART; k0 += ncw * kU) {
          float4 v[kU];
#pragma unroll
          for (int u = 0; u < kU; ++u) {
            const int k = k0 + u * ncw;
            v[u] = k < NPART ? __ldcg(reinterpret_cast<const float4*>(P + (size_t)k * m))
                             : make_float4(0.f, 0.f, 0.f, 0.f);
          }
#pragma unroll
          for (int u = 0; u < kU; ++u) {
            acc.x += v[u].x;
            acc.y += v[u].y;
            acc.z += v[u].z;
            acc.w += v[u].w;
          }
        }
      }
      if (sload) scal[t] = sreg;
      if (first && want_s)  // CTAs of fewer than 2·G threads (small m)
        for (int k = t + T; k < 2 * G; k += T) scal[k] = sval(k);
      red[warp * 32 + lane] = acc;
      named_barrier_or(1, T, false);
      if (first && warp == 0 && want_s) {  // lane-strided, then a butterfly: the same everywhere
        zdx = 0.0;
        for (int k = lane; k < G; k += 32) {
          S += scal[k];
          if (!SETUP) zdx += scal[G + k];
        }
        S = warp_sum(S);
        zdx = warp_sum(zdx);
      }
      if (warp == 0 && gi < g1) {
        double4 tot = red[lane];
        for (int w = 1; w < ncw; ++w) {
          const double4 r4 = red[w * 32 + lane];
          tot.x += r4.x;
          tot.y += r4.y;
          tot.z += r4.z;
          tot.w += r4.w;
        }
        const int row = 4 * gi;
        const double tv[4] = {tot.x, tot.y, tot.z, tot.w};
        if constexpr (SETUP) {
          // z = A·α and v = z − ‖α‖² (generate_v, core_proposedAMM.cuh:4-15)
          float zf[4], vf[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            zf[e] = (float)tv[e];
            vf[e] = (float)((double)zf[e] - S);
          }
          *reinterpret_cast<float4*>(b.z + row) = make_float4(zf[0], zf[1], zf[2], zf[3]);
          *reinterpret_cast<float4*>(b.v + row) = make_float4(vf[0], vf[1], vf[2], vf[3]);
        } else {
          const float4 yp = first ? epi_yp[lane] : *reinterpret_cast<const float4*>(yprev + row);
          const float xa[4] = {__fmul_rn(scale, yp.x), __fmul_rn(scale, yp.y),
                               __fmul_rn(scale, yp.z), __fmul_rn(scale, yp.w)};
          float yo[4];
          if (!amm) {
#pragma unroll
            for (int e = 0; e < 4; ++e) yo[e] = (float)tv[e];
          } else {
            const float4 ym = first ? epi_ym[lane] : *reinterpret_cast<const float4*>(b.y_memo + row);
            const float ymv[4] = {ym.x, ym.y, ym.z, ym.w};
            if (!centred) {  // previous: y_memo + A_S·tmp (core_previousAMM.cuh:225-232)
#pragma unroll
              for (int e = 0; e < 4; ++e) yo[e] = (float)((double)ymv[e] + tv[e]);
            } else {
              // y_memo + Σdx·v + z·dx in FP64, rounded (core_proposedAMM.cuh:198-212)
              const float4 vv = first ? epi_v[lane] : *reinterpret_cast<const float4*>(b.v + row);
              const float va[4] = {vv.x, vv.y, vv.z, vv.w};
#pragma unroll
              for (int e = 0; e < 4; ++e) {
                const float base = (float)(fma(sum_dx, (double)va[e], zdx) + (double)ymv[e]);
                yo[e] = (float)((double)base + (tv[e] - S));
              }
            }
          }
          *reinterpret_cast<float4*>(ynew + row) = make_float4(yo[0], yo[1], yo[2], yo[3]);
          if (mode == kExactMemo) {
            *reinterpret_cast<float4*>(b.x_memo + row) = make_float4(xa[0], xa[1], xa[2], xa[3]);
            *reinterpret_cast<float4*>(b.y_memo + row) = make_float4(yo[0], yo[1], yo[2], yo[3]);
          }
          if (first) {  // the next step's copy of these rows
            epi_yp[lane] = make_float4(yo[0], yo[1], yo[2], yo[3]);
            if (mode == kExactMemo) {
              epi_xm[lane] = make_float4(xa[0], xa[1], xa[2], xa[3]);
              epi_ym[lane] = epi_yp[lane];
            }
          }
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const double yd = (double)yo[e];
            xy = fma(yd, (double)xa[e], xy);
            yy = fma(yd, yd, yy);
            if (b.has_vstar) yv = fma(yd, first ? epi_vs[lane * 4 + e] : b.vstar[row + e], yv);
          }
        }
      }
      named_barrier_or(1, T, false);  // red is reused by the next row chunk
    }
    if constexpr (SETUP) {
      // the column statistics (get_norms, device_memory.h:34-59) from the column sums: α =
      // Σa/m (as the coefficient above), ‖A_j‖ = sqrt(Σa²), ‖A_j − α_j‖ = sqrt(Σa² −
      // mean²·m) clamped at 0 (the reference stores NaN when cancellation makes it negative)
      for (int j = q * T + t; j < b.n; j += G * T) {
        const double2 s = __ldcg(b.colsum + j);
        const double mean = s.x / (double)m;
        b.alpha[j] = (float)(s.x * inv_m);
        b.norm[j] = (float)sqrt(s.y);
        b.normp[j] = (float)sqrt(fmax(s.y - mean * mean * (double)m, 0.0));
      }
      if (q == 0 && warp == 0) {
        if (g0 >= g1) {  // no rows here (m/4 < number of CTAs): ‖α‖² is summed separately
          for (int k = lane; k < G; k += 32) S += __ldcg(b.spart64 + k);
          S = warp_sum(S);
        }
        if (lane == 0) *b.alpha2 = S;
      }
      xsettle();
      return;
    } else {
      if (warp == 0) {
        xy = warp_sum(xy);
        yy = warp_sum(yy);
        yv = warp_sum(yv);
        if (lane == 0) {
          b.rpart[4 * q + 0] = xy;
          b.rpart[4 * q + 1] = yy;
          b.rpart[4 * q + 2] = yv;
        }
      } else if (i + 1 < a.iter_end) {
        // the coefficient slice of the predicted next list, copied ahead (checked in prepare)
        const bool smp = nx_s[3] != 0;
        if (smp) {
          const int nslot = nx_s[1];
          const int64_t nlo = nxlo_s;
          const int nnb = nx_s[2];
          for (int k = t - 32; k < nnb; k += T - 32) {
            cp_async4(wl_idx + k, b.wl_col[nslot] + nlo + k);
            cp_async4(wl_w + k, b.wl_wm[nslot] + nlo + k);
            cp_async4(wl_al + k, b.wl_al[nslot] + nlo + k);
          }
        }
        if (t == 32) wlkey_s = smp ? nx_s[1] : -2;
      }
      named_barrier_or(1, T, false);  // this CTA's Rayleigh shares are written
      if (t == 0) bar_ok = grid_barrier(b.ticket + 2, (uint32_t)G);
      if (named_barrier_or(1, T, !bar_ok)) {
        xsettle();
        drain();
        if (t == 0) atomicOr(b.status, (uint32_t)kDevTimeout);
        return;
      }
      // λ and the next step, formed by warp 0 from the CTA shares (summed lane-strided and then
      // by an xor butterfly: the same order in every CTA); the shares reach shared memory (the
      // row-reduction scratch, free now) with one load per thread, one L2 round trip
      double* shares = reinterpret_cast<double*>(red);
      for (int k = t; k < 3 * G; k += T) shares[k] = __ldcg(b.rpart + 4 * (k / 3) + k % 3);
      named_barrier_or(1, T, false);
      if (warp == 0) {
        xy = 0.0;
        yy = 0.0;
        yv = 0.0;
        for (int k = lane; k < G; k += 32) {
          xy += shares[3 * k + 0];
          yy += shares[3 * k + 1];
          yv += shares[3 * k + 2];
        }
        xy = warp_sum(xy);
        yy = warp_sum(yy);
        yv = warp_sum(yv);
        if (lane == 0) {
          StepScalars sc;
          nxs_s = next_state(cc, i, st_s, xy, yy, yv, &sc);
          if (q == 0) record_step(b, cc, i, st_s, sc);
        }
      }
      named_barrier_or(1, T, false);  // nxs_s
      const IterState nx = nxs_s;
      if (i + 1 < a.iter_end && !nx.done) prepare(i + 1, nx);  // uniform over the grid
      if (t == 0) st_s = nx;  // published by the barrier at the top of the next step
    }
  }
  // past the last step of the launch (or the early stop): the state the next launch (or the
  // call's end) reads, and no copy still in flight
  if (!SETUP) {
    xsettle();
    drain();
    if (q == 0 && t == 0) b.st[a.iter_end & 1] = st_s;
  }
}

// ------------------------------------------------------------------------------------------
// Geometry and launch
// ------------------------------------------------------------------------------------------

using KernelFn = void (*)(PanelArgs);

// Supported (R, GC) instantiations; rows per thread = R*E.
static KernelFn pick_kernel(int dtype, int R, int GC, bool setup) {
#define AMM_PICK(EL, RR, GG)                                                     \
  if (R == RR && GC == GG)                                                       \
    return setup ? panel_kernel<EL, RR, GG, true> : panel_kernel<EL, RR, GG, false>;
  if (dtype == 1) {
    AMM_PICK(__nv_bfloat16, 1, 8)
    AMM_PICK(__nv_bfloat16, 1, 4)
    AMM_PICK(__nv_bfloat16, 2, 4)
    AMM_PICK(__nv_bfloat16, 2, 2)
    AMM_PICK(__nv_bfloat16, 4, 2)
    AMM_PICK(__nv_bfloat16, 4, 1)
  } else {
    AMM_PICK(float, 1, 8)
    AMM_PICK(float, 1, 4)
    AMM_PICK(float, 2, 4)
    AMM_PICK(float, 2, 2)
    AMM_PICK(float, 4, 2)
    AMM_PICK(float, 4, 1)
    AMM_PICK(float, 8, 1)
  }
#undef AMM_PICK
  return nullptr;
}

static cudaError_t configure(const PanelGeom& g, bool setup, KernelFn* fn, int* smem) {
  *fn = pick_kernel(g.dtype, g.slots, g.gc, setup);
  if (!*fn) return cudaErrorInvalidValue;
  *smem = smem_layout(g, setup).total;
  return cudaFuncSetAttribute(*fn, cudaFuncAttributeMaxDynamicSharedMemorySize, *smem);
}

static int env_int(const char* name, int dflt) {
  const char* v = getenv(name);
  return (v && *v) ? atoi(v) : dflt;
}

int panel_cluster_request() { return env_int("AMM_PANEL_CLUSTER", 1); }

// Rows per thread, columns per group and stages for (m, dtype): one persistent CTA per SM.
// Tuning overrides: AMM_PANEL_GC, AMM_PANEL_STAGES (0 = automatic).  With cluster > 1 the grid
// is fixed by panel_coresident (the clusters that fit at once, at least half the SMs); the
// work-list capacity is sized for that lower bound.
bool panel_geometry(int m, int dtype, int c, int n, int nsm, int cluster, PanelGeom* g) {
  const int es = dtype == 1 ? 2 : 4;
  const int E = 16 / es;
  if (m <= 0 || m % E != 0) return false;
  const int nvec = m / E;
  const int rmax = dtype == 1 ? 4 : 8;  // 32 rows per thread at most (register budget)
  int R = 1;
  while ((nvec + R - 1) / R > kMaxThreads && R < rmax) R <<= 1;
  if ((nvec + R - 1) / R > kMaxThreads) return false;
  // prefer >= 4 rows per thread so that small matrices still use few warps efficiently
  const int T = ((nvec + R - 1) / R + 31) / 32 * 32;
  const int colb = m * es;
  // ~64 KB per stage, 3 stages (one in flight while two are in use)
  int gc = 65536 / colb;
  if (gc < 1) gc = 1;
  if (gc > 8) gc = 8;
  int p2 = 1;
  while (p2 * 2 <= gc) p2 <<= 1;
  gc = p2;
  const int fgc = env_int("AMM_PANEL_GC", 0);
  if (fgc > 0) gc = fgc;
  const int stage = gc * colb;
  const int maxlist = c < n ? c : n;
  if (nsm > kMaxGrid) nsm = kMaxGrid;
  // clusters: the partial y (m floats) must fit one stage, and the ranks' row slices be whole
  // float4 groups
  if (cluster != 2 && cluster != 4 && cluster != 8) cluster = 1;
  if (cluster > 1 && (stage < 4 * m || (m / 4) % cluster != 0 || nsm < 2 * cluster))
    cluster = 1;
  const int grid_min = cluster > 1 ? nsm / 2 : nsm;
  // the stages take what the rest of the carve leaves of the budget (at most 8)
  PanelGeom probe{};
  probe.gc = gc;
  probe.wl_cap = (maxlist + grid_min - 1) / grid_min + 1;
  const int rest = smem_layout(probe, true).total;
  int ns = (kSmemBudget - rest) / stage;
  if (ns > 8) ns = 8;
  const int fns = env_int("AMM_PANEL_STAGES", 0);
  if (fns > 0 && fns < ns) ns = fns;
  if (ns < 3 || !pick_kernel(dtype, R, gc, false)) return false;
  PanelGeom b{};
  b.dtype = dtype;
  b.cluster = cluster;
  b.rows = m;
  b.nclusters = nsm / cluster;
  b.grid = b.nclusters * cluster;
  b.threads = T;
  b.slots = R;
  b.elems = E;
  b.colbytes = colb;
  b.gc = gc;
  b.nstages = ns;
  b.stage_bytes = stage;
  b.stage_area = ns * stage;
  b.wl_cap = probe.wl_cap;
  b.smem_bytes = smem_layout(b, true).total;
  *g = b;
  return b.smem_bytes <= kSmemBudget;
}

// ---- co-residency of the persistent grids ----
// The step kernel and the set-up pass synchronise all their CTAs with grid barriers, so every
// CTA of the grid (one per SM) must be resident at once.  panel_coresident checks at context
// creation that one CTA of each variant fits on an SM with its shared-memory carve; at launch
// the grids also carry the cooperative attribute, with which the runtime refuses a grid that
// cannot be co-resident (fewer SMs available to this process, e.g. under an MPS thread limit)
// instead of letting the barriers run into their time limit.  Whether the runtime accepts the
// cooperative attribute beside programmatic stream serialization is probed once per device
// with an empty kernel; where it does not, the step grids keep programmatic dependent launch
// and rely on the creation-time check.
__global__ void coop_probe_kernel() {}

static int g_coop_pdl[64] = {};  // per device: 0 unknown, 1 accepted, 2 refused

static bool coop_with_pdl() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return false;
  if (g_coop_pdl[dev] == 0) {
    cudaStream_t ps = nullptr;
    bool ok = cudaStreamCreateWithFlags(&ps, cudaStreamNonBlocking) == cudaSuccess;
    if (ok) {
      cudaLaunchConfig_t cfg{};
      cfg.gridDim = dim3(1);
      cfg.blockDim = dim3(32);
      cfg.stream = ps;
      cudaLaunchAttribute at[2];
      at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
      at[0].val.programmaticStreamSerializationAllowed = 1;
      at[1].id = cudaLaunchAttributeCooperative;
      at[1].val.cooperative = 1;
      cfg.attrs = at;
      cfg.numAttrs = 2;
      ok = cudaLaunchKernelEx(&cfg, coop_probe_kernel) == cudaSuccess;
      ok = (cudaStreamSynchronize(ps) == cudaSuccess) && ok;
      cudaStreamDestroy(ps);
    }
    cudaGetLastError();  // a refused launch leaves a (non-sticky) error behind
    g_coop_pdl[dev] = ok ? 1 : 2;
  }
  return g_coop_pdl[dev] == 1;
}

bool panel_coresident(PanelGeom* g, int nsm) {
  if (nsm > kMaxGrid) nsm = kMaxGrid;
  int fit = nsm / g->cluster;  // clusters resident at once, over both variants
  for (int setup = 0; setup < 2; ++setup) {
    KernelFn fn;
    int smem = 0;
    if (configure(*g, setup != 0, &fn, &smem) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, g->threads, (size_t)smem) !=
        cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    if (per_sm < 1) return false;
    if (g->cluster > 1) {
      cudaLaunchConfig_t cfg{};
      cfg.gridDim = dim3(g->cluster * (nsm / g->cluster));
      cfg.blockDim = dim3(g->threads);
      cfg.dynamicSmemBytes = (size_t)smem;
      cudaLaunchAttribute at[1];
      at[0].id = cudaLaunchAttributeClusterDimension;
      at[0].val.clusterDim.x = g->cluster;
      at[0].val.clusterDim.y = 1;
      at[0].val.clusterDim.z = 1;
      cfg.attrs = at;
      cfg.numAttrs = 1;
      int nc = 0;
      if (cudaOccupancyMaxActiveClusters(&nc, (void*)fn, &cfg) != cudaSuccess) {
        cudaGetLastError();
        return false;
      }
      fit = std::min(fit, nc);
    }
  }
  if (g->cluster > 1) {
    if (fit * g->cluster < nsm / 2) return false;  // the work lists are sized for >= nsm/2 CTAs
    g->nclusters = fit;
    g->grid = fit * g->cluster;
  }
  return true;
}

static cudaError_t launch_panel(const PanelArgs& a, bool setup, cudaStream_t s) {
  KernelFn fn;
  int smem = 0;
  cudaError_t e = configure(a.g, setup, &fn, &smem);
  if (e != cudaSuccess) return e;
  // step grids: programmatic dependent launch (AMM_PDL=0 turns it off, for comparison)
  static const bool pdl = env_int("AMM_PDL", 1) != 0;
  const bool dep = !setup && pdl;
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(a.g.grid);
  cfg.blockDim = dim3(a.g.threads);
  cfg.dynamicSmemBytes = (size_t)smem;
  cfg.stream = s;
  cudaLaunchAttribute at[3];
  int na = 0;
  if (dep) {
    at[na].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[na].val.programmaticStreamSerializationAllowed = 1;
    ++na;
  }
  if (a.g.cluster > 1) {
    // clusters: the grid is the clusters that fit at once (panel_coresident)
    at[na].id = cudaLaunchAttributeClusterDimension;
    at[na].val.clusterDim.x = a.g.cluster;
    at[na].val.clusterDim.y = 1;
    at[na].val.clusterDim.z = 1;
    ++na;
  } else if (!dep || coop_with_pdl()) {
    at[na].id = cudaLaunchAttributeCooperative;
    at[na].val.cooperative = 1;
    ++na;
  }
  cfg.attrs = at;
  cfg.numAttrs = na;
  e = cudaLaunchKernelEx(&cfg, fn, a);
  count_launch();
  return e != cudaSuccess ? e : cudaGetLastError();
}

cudaError_t launch_setup_panel(const Buffers& b, const PanelGeom& g, cudaStream_t s) {
  PanelArgs a{};
  a.b = b;
  a.g = g;
  a.iter = 0;
  a.iter_end = 1;
  return launch_panel(a, true, s);
}

cudaError_t launch_iter_panel(const Buffers& b, const PanelGeom& g, const CallCfg& cc, int iter,
                              int iter_end, cudaStream_t s) {
  PanelArgs a{};
  a.b = b;
  a.g = g;
  a.cc = cc;
  a.iter = iter;
  a.iter_end = iter_end;
  return launch_panel(a, false, s);
}

}  // namespace amm
