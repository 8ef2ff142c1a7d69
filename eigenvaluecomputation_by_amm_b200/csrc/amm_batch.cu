// Batched power method: λ_max of C_b = A_b·A_bᵀ for many independent FP32 matrices of uneven
// sizes in ONE persistent launch (block power iteration with K vectors and Rayleigh–Ritz), and
// the batched backward ∂λ/∂A = 2·v(vᵀA).
//
// The reference handles one matrix per run (AMM.cu:74-95); this path batches the exact product
// of powerMethod_by_exact.cuh:37-53 with the Rayleigh step of dotProduct_and_generate_x
// (common.h:103-153) generalised to a block of K orthonormal vectors.
//
// Work split: one CTA (512 threads) per matrix at a time, matrices taken largest-first from an
// atomic queue.  A matrix of m rows is held by "teams" of P threads (P = smallest power of two
// >= m/4, at least 32), each thread owning 4 consecutive rows of the K vectors X and of the
// product Y in registers; the 512/P teams split the columns.  Per group of GC columns a team
// reads the columns once (coalesced 16-byte cp.async copies into a per-thread shared-memory
// ring that keeps two or more groups in flight), forms the K·GC partial dots A_jᵀX over its
// rows, reduces them across the team (warp butterfly, then shared memory for teams wider than a
// warp) and accumulates Y += A_j·(A_jᵀX): the fused single-pass product of the main kernel.
// Exact batches of 8 vectors take a tensor-core form of the same product instead (TF32
// mma.sync with a hi + lo split, column tiles copied by TMA; see batch_kernel).
// After the pass the team partials of Y are summed in a fixed order, the Gram matrices
// G = YᵀY and H = XᵀY are reduced in FP64, X <- Y·R⁻¹ (Cholesky QR), and every rr_period
// iterations (and at the end) H is diagonalised by a warp-parallel cyclic Jacobi in FP64: its
// largest eigenvalue is λ_max, its eigenvector q gives v = X·q.

#include <cooperative_groups.h>
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <tuple>
#include <cstdint>
#include <cstring>
#include <map>
#include <vector>

#include "amm.h"
#include "amm_device.cuh"
#include "amm_internal.h"

namespace amm {
namespace batch {

constexpr int kThreads = 512;
constexpr int kWarps = kThreads / 32;
constexpr int kMaxRows = 4 * kThreads;  // 2048
constexpr int kMaxK = 8;
constexpr int kJacobiSweeps = 16;

constexpr int kMaxCols = 8192;   // AMM mode: the CDF lives in shared memory
constexpr int kVrSlot = 3;       // VR scratch per CTA: X_memo, Y_memo, saved X
constexpr int kMaxPicks = 1024;  // AMM mode: c <= n / 8

struct Mat {
  const float* A;  // column-major, ld % 4 == 0, 16-byte aligned
  int64_t ld;
  int32_t m, n;
  int64_t out_off;  // first row of this matrix's vector in the output
  int64_t st_off;   // AMM mode: first of this matrix's c xorshift states
  int32_t c;        // AMM mode: samples per product (0: exact)
  int32_t pad;
};

struct Args {
  const Mat* mats;
  const int32_t* order;  // processing order (largest first), shared by the launches of a run
  int32_t count;
  int32_t max_iter;
  double tol;
  int32_t rr_period;
  int32_t count0;        // matrices of this launch's own list, taken before the shared one
  const int32_t* order0;
  uint64_t seed;
  uint32_t* states;  // AMM mode: xorshift32 states of every matrix (advanced in place)
  uint32_t* queue;  // [0]: next item of the shared list, [1]: of the own list; zero at the start
  double* lam;      // count x K Ritz values, descending ([0] = λ_max)
  float* vec;       // Σ m: v of each matrix (top Ritz vector, unit)
  int32_t* iters;   // iterations run (-1: rank-deficient block, no result)
  // AMM mode with variance reduction: product p is exact, and memoised, when
  // (p + 1) % vr_period == 0 and for the last product; the others estimate
  // C·X = Y_memo·S + Ĉ·(X − X_memo·S), S = X_memoᵀ·X (0: no variance reduction)
  int32_t vr_period;
  int32_t vr_base;   // first slot of this launch's CTAs in vr_mem (the second launch of a run
                     // is offset past the first one's CTAs)
  float* vr_mem;     // per CTA slot: X_memo, Y_memo, then X saved while a sampled product
                     // multiplies D in its place; kMaxRows x K floats each ([row][v])
  // optional record for parity checks (null: none): each matrix's FP32 CDF at col_start[mi]
  // and the raw picks of its AMM product p < rec_products at st_off·rec_products + p·c + k
  float* rec_cdf;
  uint32_t* rec_picks;
  int32_t rec_products;
  const int64_t* col_start;
  // tensor-core kernel: one tensor map per matrix (FP32 {m rows, n columns}, 32 x 8 boxes,
  // 128-byte swizzle, zero fill outside the matrix), encoded on the host
  const CUtensorMap* tmaps;
};

// A shared-memory float4 load the compiler keeps in place (X is re-read per column group
// instead of being held in registers across the pass).
__device__ __forceinline__ float4 lds_f4(const float* p) {
  float4 v;
  asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];"
               : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
               : "r"((uint32_t)__cvta_generic_to_shared(p)));
  return v;
}

// Tensor-core product (exact mode, 8 vectors): X is stored [v][row] with a row stride of 2064
// floats (516 16-byte chunks, 4 mod 8: the 16-byte fragment loads of vector pairs land on
// disjoint banks).
constexpr int kXsStrideTC = kMaxRows + 16;

// Shared-memory position of X[row][v].  For an even block the vectors are interleaved in pairs
// ([v/2][row][2]) so that a thread's 4 rows of a vector pair are two 16-byte loads holding the
// float2 operands of the packed FMAs; the tensor-core kernel keeps [v][row].
template <int K, bool TC = false>
__device__ __forceinline__ int xs_idx(int v, int row) {
  if constexpr (TC)
    return v * kXsStrideTC + row;
  else if constexpr (K % 2 == 0)
    return (v >> 1) * (2 * kMaxRows) + row * 2 + (v & 1);
  else
    return v * kMaxRows + row;
}

// Start block: a counter-based hash of (seed, matrix, row, vector) -> uniform [-1, 1).
__device__ __forceinline__ float start_value(uint64_t seed, int mi, int row, int v) {
  uint64_t z = seed ^ (0x9E3779B97F4A7C15ull * (uint64_t)(mi + 1)) ^
               ((uint64_t)row << 20) ^ ((uint64_t)v << 52);
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return (float)(int32_t)(uint32_t)(z >> 32) * (1.0f / 2147483648.0f);
}

// Pair (p, q), p < q, of slot s in round r of a round-robin over K (even) indices.
__device__ __forceinline__ void rr_pair(int K, int r, int s, int* p, int* q) {
  int a, b;
  if (s == 0) {
    a = K - 1;
    b = r;
  } else {
    a = (r + s) % (K - 1);
    b = (r - s + (K - 1)) % (K - 1);
  }
  *p = a < b ? a : b;
  *q = a < b ? b : a;
}

// Cyclic Jacobi on the symmetric K x K matrix H (FP64, shared memory) by one warp; V receives
// the eigenvectors (columns), H the eigenvalues on its diagonal.  Rotations of one round act on
// disjoint index pairs, so a round is applied in parallel: lane = pair slot * K + index.
template <int K>
__device__ void jacobi_warp(double* H, double* V, double* cs, int lane) {
  for (int i = lane; i < K * K; i += 32) V[i] = (i / K == i % K) ? 1.0 : 0.0;
  __syncwarp();
  if constexpr (K == 1) return;
  for (int sweep = 0; sweep < kJacobiSweeps; ++sweep) {
    double off = 0.0, dia = 0.0;
    for (int i = lane; i < K * K; i += 32) {
      const double h = H[i];
      if (i / K == i % K)
        dia += h * h;
      else
        off += h * h;
    }
    off = warp_sum(off);
    dia = warp_sum(dia);
    // off-diagonal entries below ~1e-13 of the matrix: the eigenvalue error left is their
    // square over the gap (the FP64 rounding floor of `off` is ~K²·eps²·dia, so a tighter test
    // would never be met and run every sweep); also stops on NaN
    if (!(off > 1e-26 * dia)) break;
    for (int r = 0; r < K - 1; ++r) {
      if (lane < K / 2) {
        int p, q;
        rr_pair(K, r, lane, &p, &q);
        const double hpq = H[p * K + q];
        double c = 1.0, s = 0.0;
        if (hpq != 0.0) {
          // t = tan θ = sign(d)·b / (|d| + sqrt(d² + b²)), d = h_qq − h_pp, b = 2·h_pq (the
          // annihilating angle), to FP32 accuracy from d and b scaled by an exact power of two
          // (max(|d|, |b|) in [1, 2)); (c, s) = (1, t)/sqrt(1 + t²) in FP32, then two Newton
          // steps x <- x·(3 − (c² + s²))/2 in FP64 make the rotation orthogonal to FP64
          // rounding.  An angle off by FP32 rounding leaves h_pq at ~1e-7 of its size instead of
          // 0, which the next sweep removes; the eigenvalues depend only on the orthogonality.
          const double dd = H[q * K + q] - H[p * K + p], bb = 2.0 * hpq;
          const double mx = fmax(fabs(dd), fabs(bb));
          const int ex = (int)((__double_as_longlong(mx) >> 52) & 0x7ff);
          const double sc = __longlong_as_double((long long)(2046 - min(ex, 2045)) << 52);
          const float df = (float)(dd * sc), bf = (float)(bb * sc);
          const float tf = copysignf(1.f, df) *
                           __fdividef(bf, fabsf(df) + sqrtf(fmaf(df, df, bf * bf)));
          const float cf = rsqrtf(fmaf(tf, tf, 1.f));
          c = (double)cf;
          s = (double)(tf * cf);
#pragma unroll
          for (int nw = 0; nw < 2; ++nw) {
            const double f = fma(-0.5, fma(c, c, s * s), 1.5);
            c *= f;
            s *= f;
          }
        }
        cs[2 * lane] = c;
        cs[2 * lane + 1] = s;
      }
      __syncwarp();
      const int slot = lane / K, i = lane % K;
      int p = 0, q = 0;
      double c = 1.0, s = 0.0;
      const bool act = slot < K / 2;
      if (act) {
        rr_pair(K, r, slot, &p, &q);
        c = cs[2 * slot];
        s = cs[2 * slot + 1];
      }
      // columns p, q of H and V: H <- H·J, V <- V·J
      double hip = 0, hiq = 0, vip = 0, viq = 0;
      if (act) {
        hip = H[i * K + p];
        hiq = H[i * K + q];
        vip = V[i * K + p];
        viq = V[i * K + q];
      }
      __syncwarp();
      if (act) {
        H[i * K + p] = c * hip - s * hiq;
        H[i * K + q] = s * hip + c * hiq;
        V[i * K + p] = c * vip - s * viq;
        V[i * K + q] = s * vip + c * viq;
      }
      __syncwarp();
      // rows p, q: H <- Jᵀ·H
      double hpi = 0, hqi = 0;
      if (act) {
        hpi = H[p * K + i];
        hqi = H[q * K + i];
      }
      __syncwarp();
      if (act) {
        H[p * K + i] = c * hpi - s * hqi;
        H[q * K + i] = s * hpi + c * hqi;
      }
      __syncwarp();
    }
  }
}

constexpr int align16(int x) { return (x + 15) & ~15; }
constexpr int align1024(int x) { return (x + 1023) & ~1023; }
constexpr int cmax(int a, int b) { return a > b ? a : b; }

// The column ring of the product pass: every thread copies its own 16 bytes of each column of
// a group (cp.async, no register staging) RingStages<GC> groups ahead and reads back only what it
// copied, so the ring needs no barrier.  96 KB: 64 KB in flight per SM at NST = 3.
constexpr int kRingBytes = 96 * 1024;
template <int GC>
struct Ring {
  static constexpr int stages = kRingBytes / (kThreads * GC * 16);
};

// Tensor-core product: per warp and stage, 8 columns x 128 rows (4 KB, four 32 x 8 TMA boxes);
// two stages.
constexpr int kTcCols = 8;
constexpr int kTcWarpFloats = kTcCols * 128;
constexpr int kTcStageFloats = kWarps * kTcWarpFloats;

template <int K, bool TC = false>
struct Smem {
  // byte offsets into dynamic shared memory, each 16-byte aligned
  static constexpr int part = 0;                  // float [2][kWarps][32] (TC: float2 per lane)
  static constexpr int bcast = align16(part + 2 * kWarps * 32 * 4 * (TC ? 2 : 1));
                                                                         // float [kWarps][32]
  static constexpr int gpart = align16(bcast + kWarps * 32 * 4);         // double [kWarps][2*K*K]
  static constexpr int gram = align16(gpart + kWarps * 2 * K * K * 8);   // double G[K*K], H[K*K]
  static constexpr int vmat = align16(gram + 2 * K * K * 8);             // double V[K*K]
  static constexpr int rinv = align16(vmat + K * K * 8);                 // float Rinv[K*K]
  static constexpr int qv = align16(rinv + K * K * 4);                   // float q[K]
  static constexpr int cs = align16(qv + K * 4);                         // double cs[kMaxK]
  static constexpr int ritz = align16(cs + kMaxK * 8);                   // double θ[K], λ
  static constexpr int ctl = align16(ritz + (kMaxK + 1) * 8);            // int [4]
  static constexpr int tbar = align16(ctl + 16);  // uint64 [kWarps][2]: tensor-core tile copies
  static constexpr int xs = align16(tbar + kWarps * 2 * 8);              // float X[K][kMaxRows]
  static constexpr int xs_bytes = K * (TC ? kXsStrideTC : kMaxRows) * 4;
  // one region used in turn by: the column ring during a product pass; the team partials of Y
  // after it (yred); the block D of a sampled product with variance reduction (yred, during
  // that product, which then keeps its columns in registers); the pick histogram of an AMM draw
  // (hist, zeroed at the start of every draw)
  // (tensor-core kernel: 1024-byte aligned, as the 128-byte swizzle of its tile copies needs)
  static constexpr int region = TC ? align1024(xs + xs_bytes) : align16(xs + xs_bytes);
  static constexpr int yred = region;                                    // float [4*kThreads][K]
  static constexpr int hist = align16(yred + 4 * kThreads * K * 4);      // uint32 [kMaxCols]
  static constexpr int region_bytes =
      TC ? cmax(2 * kTcStageFloats * 4, 4 * kThreads * K * 4)
         : cmax(hist + kMaxCols * 4 - region, kRingBytes);
  static constexpr int total = align16(region + region_bytes);           // exact mode ends here
  static constexpr int cdf = total;                                      // float [kMaxCols]
  static constexpr int lcol = align16(cdf + kMaxCols * 4);               // int32 [kMaxPicks]
  static constexpr int lw = align16(lcol + kMaxPicks * 4);             // float [kMaxPicks]
  static constexpr int scan = align16(lw + kMaxPicks * 4);             // uint32 [40], double[32]
  static constexpr int svr = align16(scan + 40 * 4 + 32 * 8);           // float S[K*K] (VR)
  static constexpr int total_amm = align16(svr + K * K * 4);
  static_assert(gpart % 8 == 0 && cs % 8 == 0 && xs % 16 == 0 && region % 16 == 0,
                "shared-memory alignment");
  static_assert(!TC || total <= 227 * 1024, "the tensor-core layout exceeds a CTA's shared memory");
};

// One m16n8k8 TF32 tensor-core product D += A·B (FP32 accumulators), fragments as in the PTX
// ISA: lane = 4·g + t holds A(g, t), A(g+8, t), A(g, t+4), A(g+8, t+4), B(t, g), B(t+4, g) and
// D(g, 2t), D(g, 2t+1), D(g+8, 2t), D(g+8, 2t+1).
__device__ __forceinline__ void mma_tf32(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2,
                                         uint32_t a3, uint32_t b0, uint32_t b1) {
  asm("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0, %1, %2, %3}, "
      "{%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// x = hi + lo with hi x rounded to TF32 (11 significant bits, to nearest, ties away: add half
// an ulp of TF32 to the bit pattern, then clear the 13 low bits) and lo = x - hi, exact in
// FP32; the tensor core reads lo to 11 bits, so hi + lo carries x to about 2^-21 relative.
__device__ __forceinline__ void tf32_split(float x, uint32_t& hi, uint32_t& lo) {
  const uint32_t h = (__float_as_uint(x) + 0x1000u) & 0xffffe000u;
  hi = h;
  lo = __float_as_uint(x - __uint_as_float(h));
}


// Sum of the NV values d over the team (P threads).  Returns, in every lane, the total of value
// lane / (32 / NV); the caller gathers value i from lane i·(32 / NV).  Fixed reduction order
// (deterministic).
template <int NV>
__device__ __forceinline__ float team_allreduce(float (&d)[NV], float* part, int buf, int warp,
                                                int lane, int P, int team, int team_warp0) {
  float r = warp_reduce_multi<float, NV>(d, lane);
  if (P > 32) {
    float* pb = part + buf * kWarps * 32;
    pb[warp * 32 + lane] = r;
    named_barrier_or(1 + team, P, false);
    float s = 0.f;
    for (int w = 0; w < P / 32; ++w) s += pb[(team_warp0 + w) * 32 + lane];
    r = s;
  }
  return r;
}

// Rayleigh–Ritz (every rr_period steps and at the end) and the next basis, by warp 0; kept out
// of line so that its FP64 scratch does not compete for registers with the product loop.
// H = XᵀCX is diagonalised (θ, V); λ = max θ, its Ritz vector v = X·q (q and the sorted θ go
// to shared memory for the residual test the whole CTA runs next).  The next basis is
// X <- Y·M, M = V·L⁻ᵀ with L·Lᵀ = VᵀGV: Cholesky QR of the block rotated into the Ritz basis,
// so the next H is nearly diagonal and the Jacobi sweeps are few.  ctl[1]: 0 go on, 2 failed
// (rank-deficient block or a non-finite λ); ctl[2]: a Ritz pair was formed.
template <int K>
__device__ __noinline__ void ritz_step(const Args& a, int mi, int it, double* Gm, double* Hm,
                                       double* Vm, double* cs, double* ritz, float* Rinv,
                                       float* qv, int* ctl, double* scratch, int lane,
                                       bool writer, bool force_rr) {
  const bool first = (it == 0);
  const bool rr = !first && ((K == 1) || ((it % a.rr_period) == 0) || (it >= a.max_iter) ||
                             force_rr);
  if (rr) jacobi_warp<K>(Hm, Vm, cs, lane);
  // the Ritz values (lane 0: K entries)
  int st = 0;
  if (lane == 0) {
    ctl[2] = rr ? 1 : 0;
    if (rr) {
      int best = 0;
      for (int i = 1; i < K; ++i)
        if (Hm[i * K + i] > Hm[best * K + best]) best = i;
      const double lam = Hm[best * K + best];
      for (int i = 0; i < K; ++i) qv[i] = (float)Vm[i * K + best];
      double th[kMaxK];  // Ritz values, descending
      for (int i = 0; i < K; ++i) th[i] = Hm[i * K + i];
      for (int i = 0; i < K; ++i)
        for (int j = i + 1; j < K; ++j)
          if (th[j] > th[i]) {
            const double tmp = th[i];
            th[i] = th[j];
            th[j] = tmp;
          }
      for (int i = 0; i < K; ++i) ritz[i] = th[i];
      ritz[kMaxK] = lam;
      if (!isfinite(lam)) st = 2;
    }
  }
  st = __shfl_sync(0xffffffffu, st, 0);
  // The next basis, by the whole warp with the K x K matrices in shared memory (`scratch`:
  // 4·K² doubles); each entry is summed in the same order as a sequential loop would.
  double* Gp = scratch;              // VᵀGV (or G)
  double* T = scratch + K * K;       // G·V
  double* L = scratch + 2 * K * K;   // Cholesky factor (lower)
  double* Li = scratch + 3 * K * K;  // L⁻¹ (lower)
  if (st == 0) {
    if (rr) {
      for (int idx = lane; idx < K * K; idx += 32) {
        const int i = idx / K, j = idx % K;
        double acc = 0.0;
        for (int k = 0; k < K; ++k) acc += Gm[i * K + k] * Vm[k * K + j];
        T[idx] = acc;
      }
      __syncwarp();
      for (int idx = lane; idx < K * K; idx += 32) {
        const int i = idx / K, j = idx % K;
        double acc = 0.0;
        for (int k = 0; k < K; ++k) acc += Vm[k * K + i] * T[k * K + j];
        Gp[idx] = acc;
      }
    } else {
      for (int idx = lane; idx < K * K; idx += 32) Gp[idx] = Gm[idx];
    }
    for (int idx = lane; idx < K * K; idx += 32) L[idx] = 0.0;
    __syncwarp();
    double tr = 0.0;
    for (int i = 0; i < K; ++i) tr += Gp[i * K + i];
    bool ok = tr > 0.0 && isfinite(tr);
    // Cholesky, column by column: the diagonal by lane 0, the column below it by lanes j+1..;
    // one reciprocal square root per column gives both L_jj = d·d^(-1/2) and 1/L_jj (kept in
    // Ri, which takes T's place: T is dead once Gp is formed), so no step divides
    double* Ri = T;
    for (int j = 0; j < K && ok; ++j) {
      if (lane == 0) {
        double d = Gp[j * K + j];
        for (int k = 0; k < j; ++k) d -= L[j * K + k] * L[j * K + k];
        const bool good = d > 1e-24 * tr;
        const double r = good ? rsqrt(d) : 0.0;
        L[j * K + j] = good ? d * r : 0.0;
        Ri[j] = r;
        cs[0] = good ? 1.0 : 0.0;
      }
      __syncwarp();
      ok = cs[0] != 0.0;
      if (ok && lane > j && lane < K) {
        const int i = lane;
        double sv = Gp[i * K + j];
        for (int k = 0; k < j; ++k) sv -= L[i * K + k] * L[j * K + k];
        L[i * K + j] = sv * Ri[j];
      }
      __syncwarp();
    }
    if (!ok) {  // rank-deficient block: no result for this matrix
      st = 2;
    } else {
      // L⁻¹, column j by lane j (forward substitution)
      if (lane < K) {
        const int j = lane;
        for (int i = 0; i < K; ++i) Li[i * K + j] = 0.0;
        Li[j * K + j] = Ri[j];
        for (int i = j + 1; i < K; ++i) {
          double sv = 0.0;
          for (int k = j; k < i; ++k) sv += L[i * K + k] * Li[k * K + j];
          Li[i * K + j] = -sv * Ri[i];
        }
      }
      __syncwarp();
      // M = V·L⁻ᵀ (or L⁻ᵀ without a rotation); (L⁻ᵀ)[k][j] = Li[j][k] for k <= j
      for (int idx = lane; idx < K * K; idx += 32) {
        const int i = idx / K, j = idx % K;
        double sv = 0.0;
        if (rr) {
          for (int k = 0; k <= j; ++k) sv += Vm[i * K + k] * Li[j * K + k];
        } else {
          sv = (i <= j) ? Li[j * K + i] : 0.0;
        }
        Rinv[i * K + j] = (float)sv;
      }
    }
  }
  if (lane == 0) {
    if (st == 2 && writer) {
      for (int i = 0; i < K; ++i) a.lam[(int64_t)mi * K + i] = nan("");
      a.iters[mi] = -1;
    }
    ctl[1] = st;
  }
  __syncwarp();
}

// ---- variance reduction helpers, out of line so that their registers do not compete with the
// product loop's ----
// S = X_memoᵀ·X (FP64 sums over team 0's rows, into Svr) and D = X − X_memo·S in place of X
// (X saved to Xsave, [row][v], restored by vr_add_memo after the product); called by every
// thread of the CTA.
template <int K>
__device__ __noinline__ void vr_difference(const float* Xm, float* Xs, float* Xsave,
                                           double* gpart, float* Svr, int P, int r0, int t,
                                           int warp, int lane, int team) {
  const int tw = P / 32;  // warps of team 0
  if (warp < tw) {
    for (int ab = 0; ab < K * K; ++ab) {
      const int va = ab / K, vb = ab % K;
      double sv = 0.0;
#pragma unroll
      for (int e = 0; e < 4; ++e)
        sv = fma((double)Xm[(r0 + e) * K + va], (double)Xs[xs_idx<K>(vb, r0 + e)], sv);
      sv = warp_sum(sv);
      if (lane == 0) gpart[warp * K * K + ab] = sv;
    }
  }
  __syncthreads();
  if (t < K * K) {
    double sv = 0.0;
    for (int w = 0; w < tw; ++w) sv += gpart[w * K * K + t];
    Svr[t] = (float)sv;
  }
  __syncthreads();
  if (team == 0) {
    for (int e = 0; e < 4; ++e) {
      float xm[K];
#pragma unroll
      for (int v = 0; v < K; ++v) xm[v] = Xm[(r0 + e) * K + v];
#pragma unroll
      for (int vb = 0; vb < K; ++vb) {
        float d = Xs[xs_idx<K>(vb, r0 + e)];
        Xsave[(r0 + e) * K + vb] = d;
#pragma unroll
        for (int va = 0; va < K; ++va) d = fmaf(-xm[va], Svr[va * K + vb], d);
        Xs[xs_idx<K>(vb, r0 + e)] = d;  // this thread alone reads and writes its rows here
      }
    }
  }
  __syncthreads();
}

// Y += Y_memo·S over this thread's rows, and X back in place of D (team 0, once no team
// multiplies any more).
template <int K>
__device__ __noinline__ void vr_add_memo(float (&Y)[4][K], const float* Ym, const float* Svr,
                                         const float* Xsave, float* Xs, int r0) {
  for (int e = 0; e < 4; ++e) {
#pragma unroll
    for (int v = 0; v < K; ++v) Xs[xs_idx<K>(v, r0 + e)] = Xsave[(r0 + e) * K + v];
    float ym[K];
#pragma unroll
    for (int v = 0; v < K; ++v) ym[v] = Ym[(r0 + e) * K + v];
#pragma unroll
    for (int vb = 0; vb < K; ++vb) {
      float acc = Y[e][vb];
#pragma unroll
      for (int va = 0; va < K; ++va) acc = fmaf(ym[va], Svr[va * K + vb], acc);
      Y[e][vb] = acc;
    }
  }
}

// The memo pair (X_memo, Y_memo) <- (X, Y) over this thread's rows (team 0).
template <int K>
__device__ __noinline__ void vr_store_memo(const float (&Y)[4][K], float* Xm, float* Ym,
                                           const float* Xs, int r0) {
  for (int e = 0; e < 4; ++e)
#pragma unroll
    for (int v = 0; v < K; ++v) {
      Xm[(r0 + e) * K + v] = Xs[xs_idx<K>(v, r0 + e)];
      Ym[(r0 + e) * K + v] = Y[e][v];
    }
}

// One FP64 tensor-core product D += A·B (m8n8k4, FP64 accumulation), fragments as in the PTX
// ISA: lane = 4·g + t holds A(g, t), B(t, g), D(g, 2t) and D(g, 2t+1).
__device__ __forceinline__ void mma_f64(double (&d)[2], double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
      : "+d"(d[0]), "+d"(d[1])
      : "d"(a), "d"(b));
}

// Gram matrices of the block, G = YᵀY and H = sym(XᵀY), in FP64 over team 0's rows (the only
// team holding the summed Y, here in shared memory as Ys[row][v]); called by every thread of the
// CTA.  For 8 vectors each warp of team 0 multiplies its 128 rows on the FP64 tensor cores: per
// 4 rows one m8n8k4 product for G (A = Yᵀ, B = Y: lane 4·g + t supplies Y[row t][vector g] to
// both) and one for XᵀY (A = Xᵀ); FP32 × FP32 products are exact in FP64.  For fewer vectors
// each thread forms its FP64 partials over its 4 rows, 8 entries at a time, summed over the warp
// by one multi-value butterfly per 8 entries.  The team's warps are then summed in a fixed
// order.  Kept out of line so that its registers do not compete with the product loop's.
template <int K, bool TC>
__device__ __noinline__ void gram_step(const float* Xs, const float* Ys, double* gpart,
                                       double* Gm, double* Hm, int P, int r0, int t, int warp,
                                       int lane, int team) {
  constexpr int NP = K * (K + 1) / 2;
  const int tw = P / 32;  // warps of team 0
  if constexpr (K == 8) {
    // gpart[warp][0..63]: this warp's G (row-major), [64..127]: its XᵀY
    if (team == 0) {  // warp-uniform (P >= 32)
      __syncwarp();   // the warp's rows of Ys were written by its own lanes
      double dg[2] = {0.0, 0.0}, dh[2] = {0.0, 0.0};
      const int g = lane >> 2, tq = lane & 3;
      const int rb = 128 * warp;  // team 0's warp w holds rows [128w, 128w + 128)
#pragma unroll 4
      for (int k = 0; k < 32; ++k) {
        const int row = rb + 4 * k + tq;
        const double y = (double)Ys[row * K + g];
        const double x = (double)Xs[xs_idx<K, TC>(g, row)];
        mma_f64(dg, y, y);
        mma_f64(dh, x, y);
      }
      double* gp = gpart + warp * 2 * K * K;
      gp[g * K + 2 * tq] = dg[0];
      gp[g * K + 2 * tq + 1] = dg[1];
      gp[K * K + g * K + 2 * tq] = dh[0];
      gp[K * K + g * K + 2 * tq + 1] = dh[1];
    }
    __syncthreads();
    if (t < 2 * NP) {
      const int which = t / NP, pi = t % NP;
      int a1 = 0, rem = pi;
      while (rem >= K - a1) {
        rem -= K - a1;
        ++a1;
      }
      const int b1 = a1 + rem;
      double s = 0.0;
      if (which == 0) {
        for (int w = 0; w < tw; ++w) s += gpart[w * 2 * K * K + a1 * K + b1];
      } else {
        double sa = 0.0, sb = 0.0;
        for (int w = 0; w < tw; ++w) {
          sa += gpart[w * 2 * K * K + K * K + a1 * K + b1];
          sb += gpart[w * 2 * K * K + K * K + b1 * K + a1];
        }
        s = 0.5 * (sa + sb);
      }
      double* D = which ? Hm : Gm;
      D[a1 * K + b1] = s;
      D[b1 * K + a1] = s;
    }
    __syncthreads();
  } else {
    constexpr int NV2 = 2 * NP;        // G entries (pair index), then H entries
    constexpr int NB = (NV2 + 7) / 8;  // batches of 8 entries
    if (team == 0) {                   // warp-uniform (P >= 32)
      float y[4][K];
#pragma unroll
      for (int e = 0; e < 4; ++e)
#pragma unroll
        for (int v = 0; v < K; ++v) y[e][v] = Ys[(r0 + e) * K + v];
#pragma unroll
      for (int bt = 0; bt < NB; ++bt) {
        double d[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) d[i] = 0.0;
        int pidx = 0;
#pragma unroll
        for (int a0 = 0; a0 < K; ++a0)
#pragma unroll
          for (int b0 = a0; b0 < K; ++b0, ++pidx) {
            if (pidx / 8 == bt) {
              double gg = 0.0;
#pragma unroll
              for (int e = 0; e < 4; ++e) gg = fma((double)y[e][a0], (double)y[e][b0], gg);
              d[pidx % 8] = gg;
            }
            if ((NP + pidx) / 8 == bt) {
              double h = 0.0;
#pragma unroll
              for (int e = 0; e < 4; ++e) {
                const float xa = Xs[xs_idx<K, TC>(a0, r0 + e)];
                const float xb = Xs[xs_idx<K, TC>(b0, r0 + e)];
                h = fma(0.5 * (double)xa, (double)y[e][b0], h);
                h = fma(0.5 * (double)xb, (double)y[e][a0], h);
              }
              d[(NP + pidx) % 8] = h;
            }
          }
        const double r = warp_reduce_multi<double, 8>(d, lane);  // entry 8·bt + lane/4
        const int vi = bt * 8 + (lane >> 2);
        if ((lane & 3) == 0 && vi < NV2) gpart[warp * NV2 + vi] = r;
      }
    }
    __syncthreads();
    if (t < NV2) {
      double s = 0.0;
      for (int w = 0; w < tw; ++w) s += gpart[w * NV2 + t];
      const int which = t / NP, pi = t % NP;
      int a1 = 0, rem = pi;
      while (rem >= K - a1) {
        rem -= K - a1;
        ++a1;
      }
      const int b1 = a1 + rem;
      double* D = which ? Hm : Gm;
      D[a1 * K + b1] = s;
      D[b1 * K + a1] = s;
    }
    __syncthreads();
  }
}

template <int K, int GC, bool TC = false>
__global__ void __launch_bounds__(kThreads, 1) batch_kernel(const __grid_constant__ Args a) {
  constexpr int NV = K * GC;
  static_assert(TC || (NV <= 32 && (32 % NV) == 0), "K*GC must divide 32");
  static_assert(!TC || (K == 8 && GC == kTcCols), "the tensor-core product runs 8 vectors");
  using SL = Smem<K, TC>;
  extern __shared__ __align__(16) unsigned char smem[];
  float* yred = reinterpret_cast<float*>(smem + SL::yred);
  float* part = reinterpret_cast<float*>(smem + SL::part);
  float* bcast = reinterpret_cast<float*>(smem + SL::bcast);
  double* gpart = reinterpret_cast<double*>(smem + SL::gpart);
  double* Gm = reinterpret_cast<double*>(smem + SL::gram);
  double* Hm = Gm + K * K;
  double* Vm = reinterpret_cast<double*>(smem + SL::vmat);
  float* Rinv = reinterpret_cast<float*>(smem + SL::rinv);
  float* qv = reinterpret_cast<float*>(smem + SL::qv);
  double* cs = reinterpret_cast<double*>(smem + SL::cs);
  double* ritz = reinterpret_cast<double*>(smem + SL::ritz);
  int* ctl = reinterpret_cast<int*>(smem + SL::ctl);
  float* Xs = reinterpret_cast<float*>(smem + SL::xs);  // X, one copy for all teams: [v][row]
  float* cdf = reinterpret_cast<float*>(smem + SL::cdf);
  uint32_t* hist = reinterpret_cast<uint32_t*>(smem + SL::hist);
  int32_t* lcol = reinterpret_cast<int32_t*>(smem + SL::lcol);
  float* lw = reinterpret_cast<float*>(smem + SL::lw);
  uint32_t* scan = reinterpret_cast<uint32_t*>(smem + SL::scan);
  double* dscan = reinterpret_cast<double*>(smem + SL::scan + 40 * 4);
  float* Svr = reinterpret_cast<float*>(smem + SL::svr);
  uint64_t* tbar = reinterpret_cast<uint64_t*>(smem + SL::tbar);

  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  const int CL = (int)cluster.num_blocks();   // CTAs sharing one matrix
  const int crank = (int)cluster.block_rank();
  const bool writer = (crank == 0);           // rank 0 writes the results
  // tensor-core kernel: the warps' stage barriers of the tile copies (one arrival each: the
  // issuing lane's expect_tx).  The tiles' 128-byte swizzle is laid out for a 1024-byte aligned
  // region (true of a kernel without static shared memory); were it not, no copy is issued and
  // every matrix is reported without a result.
  uint32_t tph = 0;         // phase parity of this warp's two stages (alike in every lane)
  // no more copies in this warp (misaligned region, or a copy that timed out: the warp then
  // neither issues nor waits, so that later waits cannot time out one after another)
  bool tdead = TC && (smem_addr(smem + SL::region) & 1023u) != 0u;
  bool tfail = tdead;       // this pass's product is not to be trusted
  int tfail_mi = -1;        // the matrix of this CTA that gets no result for that reason
  if constexpr (TC) {
    if (t == 0) {
      for (int i = 0; i < 2 * kWarps; ++i) mbar_init(&tbar[i], 1);
      fence_barrier_init();
    }
    __syncthreads();
  }
  // the failure record, written once the cluster is done with the matrix (after the cluster
  // barrier of the next fetch), so that no result write of a peer comes after it
  auto record_tfail = [&]() {
    if (TC && tfail_mi >= 0 && t == 0) {
      for (int i = 0; i < K; ++i) a.lam[(int64_t)tfail_mi * K + i] = nan("");
      a.iters[tfail_mi] = -1;
    }
    tfail_mi = -1;
  };
  // a launch queued behind this one as a programmatic dependent may now take the SMs left
  griddep_launch_dependents();
  for (;;) {
    // rank 0 takes the next matrix, from this launch's own list first, then from the list it
    // shares with the other launch of the run; the cluster reads it from rank 0
    if (writer && t == 0) {
      int next = -1;
      if (a.count0 > 0) {
        const uint32_t k = atomicAdd(a.queue + 1, 1u);
        if (k < (uint32_t)a.count0) next = a.order0[k];
      }
      if (next < 0) {
        const uint32_t k = atomicAdd(a.queue, 1u);
        if (k < (uint32_t)a.count) next = a.order[k];
      }
      ctl[0] = next;
    }
    cluster.sync();
    const int mi = *cluster.map_shared_rank(&ctl[0], 0);
    cluster.sync();
    record_tfail();
    if (mi < 0) {
      // a launch queued behind another (programmatic dependent) ends only after it, so that
      // the work after it in the stream sees both; returns at once in any other launch
      griddep_wait();
      return;
    }
    const Mat M = a.mats[mi];
    const int m = M.m, n = M.n;
    int P = 32;
    while (P < kThreads && 4 * P < m) P <<= 1;
    const int NT = kThreads / P;
    const int team = t / P, tl = t % P;
    const int NTG = CL * NT;             // teams of the whole cluster split the columns
    const int gteam = crank * NT + team;
    const int team_warp0 = team * (P / 32);
    const int r0 = 4 * tl;
    const bool amm = !TC && M.c > 0;  // the tensor-core kernel runs exact batches only
    double total = 0.0;
    if (amm) {
      // ---- column norms² (get_norms, device_memory.h:34-59) into cdf[], then the CDF ----
      int buf = 0;
      for (int g0 = gteam * GC; g0 < n; g0 += NTG * GC, buf ^= 1) {
        float d[GC];
#pragma unroll
        for (int c = 0; c < GC; ++c) {
          float4 av = make_float4(0.f, 0.f, 0.f, 0.f);
          if (r0 < m && g0 + c < n)
            av = __ldg(reinterpret_cast<const float4*>(M.A + r0 + (int64_t)(g0 + c) * M.ld));
          if (r0 + 1 >= m) av.y = 0.f;
          if (r0 + 2 >= m) av.z = 0.f;
          if (r0 + 3 >= m) av.w = 0.f;
          d[c] = fmaf(av.x, av.x, fmaf(av.y, av.y, fmaf(av.z, av.z, av.w * av.w)));
        }
        const float red = team_allreduce<GC>(d, part, buf, warp, lane, P, team, team_warp0);
        if (tl < GC * (32 / GC) && (lane % (32 / GC)) == 0) {
          const int c = lane / (32 / GC);
          if (g0 + c < n) cdf[g0 + c] = red;
        }
      }
      if (CL > 1) {  // norms of the columns the other CTAs of the cluster own
        cluster.sync();
        for (int j = t; j < n; j += kThreads) {
          const int owner = ((j / GC) % NTG) / NT;
          if (owner != crank) cdf[j] = *cluster.map_shared_rank(&cdf[j], owner);
        }
        cluster.sync();  // nobody overwrites its norms before every CTA has gathered
      }
      __syncthreads();
      // inclusive prefix in FP64, stored as FP32 (set_weights / CUB scan, common.h:34-40 and
      // powerMethod_by_previous.cuh:26-32); each thread owns a run of consecutive columns
      const int per = (n + kThreads - 1) / kThreads;
      const int j0 = t * per, j1 = min(n, j0 + per);
      double run = 0.0;
      for (int j = j0; j < j1; ++j) run += (double)cdf[j];
      // block exclusive scan of the run totals (FP64, fixed order)
      double incl = run;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const double y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
      }
      if (lane == 31) dscan[warp] = incl;
      __syncthreads();
      if (warp == 0) {
        double w = lane < kWarps ? dscan[lane] : 0.0;
        double wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const double y = __shfl_up_sync(0xffffffffu, wi, o);
          if (lane >= o) wi += y;
        }
        if (lane < kWarps) dscan[lane] = wi - w;
        if (lane == 31) dscan[kWarps] = wi;
      }
      __syncthreads();
      double pre = dscan[warp] + incl - run;
      total = dscan[kWarps];
      __syncthreads();
      for (int j = j0; j < j1; ++j) {
        const float nj = cdf[j];
        pre += (double)nj;
        cdf[j] = (float)pre;  // in place: this thread alone reads and writes cdf[j0, j1)
        hist[j] = 0u;
        if (a.rec_cdf && writer) a.rec_cdf[a.col_start[mi] + j] = cdf[j];
      }
      __syncthreads();
    }
    // AMM mode with variance reduction: this CTA's memo slot (CTA-private: every thread reads
    // back only the rows it wrote) and whether it holds an exact product of this matrix
    const bool vr = amm && a.vr_period > 0;
    float* Xm = a.vr_mem + (size_t)(a.vr_base + blockIdx.x) * (kVrSlot * kMaxRows * K);
    float* Ym = Xm + kMaxRows * K;
    float* Xsave = Ym + kMaxRows * K;
    bool memo = false;
    bool prev_exact = false;  // the product the Ritz step of this iteration uses was exact

    // ---- start block X0 (hash), orthonormalised below like every later Y ----
    float Y[4][K];
#pragma unroll
    for (int e = 0; e < 4; ++e)
#pragma unroll
      for (int v = 0; v < K; ++v)
        Y[e][v] = (r0 + e < m) ? start_value(a.seed, mi, r0 + e, v) : 0.f;
    if (team == 0)
#pragma unroll
      for (int v = 0; v < K; ++v)
#pragma unroll
        for (int e = 0; e < 4; ++e) Xs[xs_idx<K, TC>(v, r0 + e)] = 0.f;
    __syncthreads();

    int it = 0, state = 0;  // state: 0 running, 1 converged / last, 2 degenerate
    for (;; ++it) {
      // ---- Gram matrices of the block: G = YᵀY, H = sym(XᵀY) (FP64, team 0's rows), from a
      // shared-memory copy of team 0's Y (each thread reads back only its own rows) ----
      if (team == 0) {
#pragma unroll
        for (int e = 0; e < 4; ++e)
#pragma unroll
          for (int v = 0; v < K; ++v) yred[(r0 + e) * K + v] = Y[e][v];
      }
      gram_step<K, TC>(Xs, yred, gpart, Gm, Hm, P, r0, t, warp, lane, team);
      // (gpart, summed into Gm and Hm above, is the Ritz step's scratch)
      if (warp == 0)
        ritz_step<K>(a, mi, it, Gm, Hm, Vm, cs, ritz, Rinv, qv, ctl, gpart, lane, writer,
                     vr && prev_exact);
      __syncthreads();
      // team 0's Y back from its shared-memory copy (not held in registers across the two
      // out-of-line steps, which then get the registers for themselves)
      if (team == 0) {
#pragma unroll
        for (int e = 0; e < 4; ++e)
#pragma unroll
          for (int v = 0; v < K; ++v) Y[e][v] = yred[(r0 + e) * K + v];
      }
      if (ctl[2] && ctl[1] == 0) {
        // residual of the top Ritz pair, r = C·v − λ·v = (Y − λ·X)·q, over team 0's rows (FP64)
        const double lam = ritz[kMaxK];
        double r2 = 0.0;
        if (team == 0 && r0 < m) {
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            float yq = 0.f, xq = 0.f;
#pragma unroll
            for (int v = 0; v < K; ++v) {
              yq = fmaf(Y[e][v], qv[v], yq);
              xq = fmaf(Xs[xs_idx<K, TC>(v, r0 + e)], qv[v], xq);
            }
            const double r = (double)yq - lam * (double)xq;
            r2 = fma(r, r, r2);
          }
        }
        r2 = warp_sum(r2);
        if (lane == 0) gpart[warp] = r2;
        __syncthreads();
        if (t == 0) {
          double s = 0.0;
          for (int w = 0; w < kWarps; ++w) s += gpart[w];
          // with variance reduction only an exact product's residual is the true one
          const bool done = (sqrt(s) <= a.tol * fabs(lam) && (!vr || prev_exact)) ||
                            it >= a.max_iter;
          if (done) {
            if (writer) {
              for (int i = 0; i < K; ++i) a.lam[(int64_t)mi * K + i] = ritz[i];
              a.iters[mi] = it;
            }
            ctl[1] = 1;
          }
        }
        __syncthreads();
      }
      state = ctl[1];
      if (state != 0) {
        if (state == 1 && team == 0 && writer) {  // v = X·q over this thread's rows
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            if (r0 + e < m) {
              float s = 0.f;
#pragma unroll
              for (int v = 0; v < K; ++v) s = fmaf(Xs[xs_idx<K, TC>(v, r0 + e)], qv[v], s);
              a.vec[M.out_off + r0 + e] = s;
            }
          }
        }
        break;
      }
      // ---- X <- Y·M (team 0 writes the shared copy) ----
      if (team == 0) {
#pragma unroll
        for (int j = 0; j < K; ++j) {
          float xj[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            float s = 0.f;
#pragma unroll
            for (int i = 0; i < K; ++i) s = fmaf(Y[e][i], Rinv[i * K + j], s);
            xj[e] = s;
          }
#pragma unroll
          for (int e = 0; e < 4; ++e) Xs[xs_idx<K, TC>(j, r0 + e)] = xj[e];
        }
      }
      __syncthreads();
      // kind of product `it`: exact in exact mode; in AMM mode with variance reduction exact
      // (and memoised) when (it + 1) % vr_period == 0 (powerMethod_by_previous.cuh:135-157)
      // and for the last product, so that the reported Ritz values come from an exact product
      const bool exact_p =
          !amm || (vr && ((it + 1) % a.vr_period == 0 || it + 1 >= a.max_iter));
      const bool wamm = amm && !exact_p;  // this product is sampled
      // ---- AMM: draw c columns (get_rand + pick_index, device_memory.h:506-545) and list the
      // distinct ones in ascending order with weight multiplicity / (c·p_j) ----
      int ncols = n;
      if (wamm) {
        // the histogram shares its memory with the column ring of the last product pass
        for (int j = t; j < n; j += kThreads) hist[j] = 0u;
        __syncthreads();
        const float total_f = cdf[n - 1];
        uint32_t* st = a.states + M.st_off;
        // every CTA of the cluster draws the same picks from the same states; rank 0 stores the
        // advanced states once all have read them
        uint32_t ys[kMaxPicks / kThreads];
#pragma unroll
        for (int u = 0; u < kMaxPicks / kThreads; ++u) {
          const int k = t + u * kThreads;
          ys[u] = k < M.c ? xorshift32(st[k]) : 0u;
        }
        if (CL > 1) cluster.sync();
#pragma unroll
        for (int u = 0; u < kMaxPicks / kThreads; ++u) {
          const int k = t + u * kThreads;
          if (k >= M.c) continue;
          const uint32_t y = ys[u];
          if (writer) st[k] = y;
          const float target = __fmul_rn(total_f, uniform_from(y));
          int lo = 0, hi = n;  // first i with cdf[i] > target, else n - 1
          while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (cdf[mid] <= target)
              lo = mid + 1;
            else
              hi = mid;
          }
          const int pick = lo < n ? lo : n - 1;
          atomicAdd(&hist[pick], 1u);
          if (a.rec_picks && writer && it < a.rec_products)
            a.rec_picks[M.st_off * a.rec_products + (int64_t)it * M.c + k] = (uint32_t)pick;
        }
        __syncthreads();
        const int per = (n + kThreads - 1) / kThreads;
        const int j0 = t * per, j1 = min(n, j0 + per);
        uint32_t nz = 0;
        for (int j = j0; j < j1; ++j) nz += hist[j] ? 1u : 0u;
        uint32_t cd = 0;
        uint32_t r = block_exclusive_scan(nz, scan, &cd);
        for (int j = j0; j < j1; ++j) {
          const uint32_t mult = hist[j];
          if (mult) {
            // the realised probability of column j is its FP32 CDF step over the total
            const double step = (double)cdf[j] - (j > 0 ? (double)cdf[j - 1] : 0.0);
            lcol[r] = j;
            lw[r] = (float)((double)mult * (double)total_f / ((double)M.c * step));
            ++r;
            hist[j] = 0u;
          }
        }
        ncols = (int)cd;
        __syncthreads();
      }
      // ---- variance reduction: S = X_memoᵀ·X (FP64 sums over team 0's rows) and the block
      // the sampled product multiplies, D = X − X_memo·S, in place of X; Y_memo·S is added,
      // and X put back, once the product is summed ----
      const bool use_d = wamm && memo;
      if (use_d) vr_difference<K>(Xm, Xs, Xsave, gpart, Svr, P, r0, t, warp, lane, team);
      const float* Xsrc = Xs;  // X, or D in its place
      // ---- Y = C·X (or its AMM estimate): the fused pass over the columns (team-local) ----
      const bool rows = r0 < m;
      int buf = 0;
      if constexpr (TC) {
        // ---- tensor-core pass (exact mode, 8 vectors).  Warp wi of a team owns the team's
        // rows [128·wi, 128·wi + 128); per group of 8 columns its lane 0 copies those rows into
        // the warp's own 4 KB tile (two stages) with four TMA boxes of 32 rows x 8 columns
        // (128-byte swizzle: 16-byte chunk q of a column's 32-row line stored at q ^ (column
        // mod 8); rows past m and columns past n arrive as zeros), completing on the stage's
        // mbarrier.  Phase 1, per 16-row block: Tᵀ(16 x 8) += [X_hi | X_lo]ᵀ·A_blk, rows 0-7 of
        // the 16 holding X_hi, rows 8-15 X_lo, once with A_hi and once with A_lo (all four split
        // terms in two products); the rows of the block are ordered so that a lane's operands are
        // 4 consecutive rows (one 16-byte load each of A and X).  The team's warps sum their T
        // (fixed order).  Phase 2, per 16-row tile: Y += A_tile·T with the 8 columns ordered
        // 0,2,4,6 | 1,3,5,7 along k, so that the lane's T values are exactly its B operand; three
        // products (A_hi·T_hi, A_hi·T_lo, A_lo·T_hi). ----
        const int W = P / 32;               // warps of the team
        const int wi = tl >> 5;             // this warp's place in the team
        const int g = lane >> 2, tq = lane & 3;
        const int rbase = 128 * wi;         // first row of this warp
        const int nblk = max(0, min(8, (m - rbase + 15) >> 4));  // 16-row blocks below m
        const int nbox = (nblk + 1) >> 1;   // 32-row boxes below m
        float* wtile = reinterpret_cast<float*>(smem + SL::region) + warp * kTcWarpFloats;
        uint64_t* wbar = tbar + 2 * warp;   // this warp's stage barriers
        const CUtensorMap* tmap = a.tmaps + mi;
        float yacc[8][4];
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) yacc[i][j] = 0.f;
        auto issue = [&](int g0, int st) {
          // (the warp's reads of the stage ended before the __syncwarp that closed the group
          // which last used it); lane 0 announces the bytes, lanes 0..nbox-1 issue a box each
          if (nbox > 0 && !tdead) {
            if (lane == 0) mbar_arrive_expect_tx(&wbar[st], (uint32_t)nbox * 1024u);
            __syncwarp();
            if (lane < nbox)
              tma_load_2d(wtile + st * kTcStageFloats + lane * 256, tmap, rbase + 32 * lane, g0,
                          &wbar[st]);
          }
        };
        // every thread's earlier accesses of the tile region (the Gram step's copy of Y, the
        // team sums of the last pass, its tiles) are ordered before the first copies' writes
        fence_proxy_async_smem();
        __syncthreads();
        const int gstep = NTG * kTcCols;
        int st = 0;
        if (gteam * kTcCols < ncols) issue(gteam * kTcCols, 0);
#pragma unroll 1
        for (int g0 = gteam * kTcCols; g0 < ncols; g0 += gstep, buf ^= 1) {
          if (g0 + gstep < ncols) issue(g0 + gstep, st ^ 1);
          if (nbox > 0 && !tdead) {  // group g0 has landed (bounded wait; a timeout marks the matrix)
            const bool ok = mbar_wait_bounded(&wbar[st], (tph >> st) & 1u);
            tph ^= 1u << st;
            if (__any_sync(0xffffffffu, !ok)) tfail = tdead = true;
          }
          const float* tile = wtile + st * kTcStageFloats;
          // phase 1: T = AᵀX over this warp's rows
          float d[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll 2
          for (int sb = 0; sb < nblk; ++sb) {
            const float4 av = lds_f4(tile + (sb >> 1) * 256 + g * 32 + 4 * ((4 * (sb & 1) + tq) ^ g));
            const float4 xv = lds_f4(Xs + g * kXsStrideTC + rbase + 16 * sb + 4 * tq);
            uint32_t ah[4], al[4], xh[4], xl[4];
            tf32_split(av.x, ah[0], al[0]);
            tf32_split(av.y, ah[1], al[1]);
            tf32_split(av.z, ah[2], al[2]);
            tf32_split(av.w, ah[3], al[3]);
            tf32_split(xv.x, xh[0], xl[0]);
            tf32_split(xv.y, xh[1], xl[1]);
            tf32_split(xv.z, xh[2], xl[2]);
            tf32_split(xv.w, xh[3], xl[3]);
            // k = tq <-> row 4·tq (+2), k = tq + 4 <-> row 4·tq + 1 (+2); the block's four
            // products start from zero and the block sums are added in FP32 with rounding to
            // nearest (the tensor core's own accumulation is not rounded to nearest, and a long
            // chain of it drifts: 1e-5 relative over a 2048-row pass)
            // (two independent chains of two, one per k-half, so that they overlap)
            float db0[4] = {0.f, 0.f, 0.f, 0.f}, db1[4] = {0.f, 0.f, 0.f, 0.f};
            mma_tf32(db0, xh[0], xl[0], xh[1], xl[1], ah[0], ah[1]);
            mma_tf32(db1, xh[2], xl[2], xh[3], xl[3], ah[2], ah[3]);
            mma_tf32(db0, xh[0], xl[0], xh[1], xl[1], al[0], al[1]);
            mma_tf32(db1, xh[2], xl[2], xh[3], xl[3], al[2], al[3]);
#pragma unroll
            for (int j = 0; j < 4; ++j) d[j] += db0[j] + db1[j];
          }
          // lane (g, tq): T[col 2·tq][v g] and T[col 2·tq + 1][v g] (hi and lo rows summed)
          float t0 = d[0] + d[2], t1 = d[1] + d[3];
          if (W > 1) {
            float2* pb = reinterpret_cast<float2*>(part) + buf * kWarps * 32;
            pb[warp * 32 + lane] = make_float2(t0, t1);
            named_barrier_or(1 + team, P, false);
            t0 = 0.f;
            t1 = 0.f;
            for (int w = 0; w < W; ++w) {
              const float2 q = pb[(team_warp0 + w) * 32 + lane];
              t0 += q.x;
              t1 += q.y;
            }
          }
          uint32_t th0, tl0, th1, tl1;
          tf32_split(t0, th0, tl0);
          tf32_split(t1, th1, tl1);
          // phase 2: Y += A·T over this warp's 16-row tiles
          const int ce = 2 * tq, co = 2 * tq + 1;  // the lane's columns
          const float* pe = tile + ce * 32 + (g & 3);
          const float* po = tile + co * 32 + (g & 3);
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            if (i >= nblk) break;
            // rows 16i + g and 16i + g + 8: box i/2, 16-byte chunks q0 and q0 + 2 of its lines
            const int q0 = 4 * (i & 1) + (g >> 2), q1 = q0 + 2;
            const int bo = (i >> 1) * 256;
            uint32_t ah[4], al[4];
            tf32_split(pe[bo + 4 * (q0 ^ ce)], ah[0], al[0]);
            tf32_split(pe[bo + 4 * (q1 ^ ce)], ah[1], al[1]);
            tf32_split(po[bo + 4 * (q0 ^ co)], ah[2], al[2]);
            tf32_split(po[bo + 4 * (q1 ^ co)], ah[3], al[3]);
            // three products from zero (small terms first), then one rounded FP32 add per
            // element into Y, which sums over every group of the pass
            float dt[4] = {0.f, 0.f, 0.f, 0.f};
            mma_tf32(dt, al[0], al[1], al[2], al[3], th0, th1);
            mma_tf32(dt, ah[0], ah[1], ah[2], ah[3], tl0, tl1);
            mma_tf32(dt, ah[0], ah[1], ah[2], ah[3], th0, th1);
#pragma unroll
            for (int j = 0; j < 4; ++j) yacc[i][j] += dt[j];
          }
          __syncwarp();  // every lane is done with this stage before it is refilled
          st ^= 1;
        }
        // (every copy issued was waited on: none can still be landing in the tiles)
        if (__syncthreads_or(tfail ? 1 : 0)) tfail_mi = mi;
        tfail = tdead;
        // the team partials of Y through yred (which shares the tiles' memory), summed over the
        // teams in a fixed order by team 0
        __syncthreads();
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          if (i >= nblk) break;
          const int row = team * 4 * P + rbase + 16 * i + g;
          *reinterpret_cast<float2*>(yred + row * K + 2 * tq) = make_float2(yacc[i][0], yacc[i][1]);
          *reinterpret_cast<float2*>(yred + (row + 8) * K + 2 * tq) =
              make_float2(yacc[i][2], yacc[i][3]);
        }
        __syncthreads();
        if (team == 0) {
#pragma unroll
          for (int e = 0; e < 4; ++e)
#pragma unroll
            for (int v = 0; v < K; ++v) {
              float s = 0.f;
              if (rows)
                for (int tm = 0; tm < NT; ++tm) s += yred[((tm * 4 * P) + r0 + e) * K + v];
              Y[e][v] = s;
            }
        }
      } else {
#pragma unroll
      for (int e = 0; e < 4; ++e)
#pragma unroll
        for (int v = 0; v < K; ++v) Y[e][v] = 0.f;
      const float* __restrict__ Ab = M.A + r0;
      // one group of GC columns (weights in AMM mode): the team's dots A_jᵀX over its rows,
      // their sums over the team, and Y += A_j·(A_jᵀX)·w_j
      auto multiply = [&](const float4 (&av)[GC], const float (&wt)[GC]) {
        float d[NV];
        if constexpr (K % 2 == 0) {
          // packed FP32x2: a vector pair per instruction (X pairs interleaved in shared memory)
#pragma unroll
          for (int vp = 0; vp < K / 2; ++vp) {
            const float4 x01 = lds_f4(Xsrc + vp * 2 * kMaxRows + 2 * r0);      // rows 0, 1
            const float4 x23 = lds_f4(Xsrc + vp * 2 * kMaxRows + 2 * r0 + 4);  // rows 2, 3
            const float2 xr[4] = {make_float2(x01.x, x01.y), make_float2(x01.z, x01.w),
                                  make_float2(x23.x, x23.y), make_float2(x23.z, x23.w)};
#pragma unroll
            for (int c = 0; c < GC; ++c) {
              float2 s = __fmul2_rn(make_float2(av[c].x, av[c].x), xr[0]);
              s = __ffma2_rn(make_float2(av[c].y, av[c].y), xr[1], s);
              s = __ffma2_rn(make_float2(av[c].z, av[c].z), xr[2], s);
              s = __ffma2_rn(make_float2(av[c].w, av[c].w), xr[3], s);
              d[c * K + 2 * vp] = s.x;
              d[c * K + 2 * vp + 1] = s.y;
            }
          }
        } else {
#pragma unroll
          for (int v = 0; v < K; ++v) {
            const float4 xv = lds_f4(Xsrc + v * kMaxRows + r0);
#pragma unroll
            for (int c = 0; c < GC; ++c) {
              float s = av[c].x * xv.x;
              s = fmaf(av[c].y, xv.y, s);
              s = fmaf(av[c].z, xv.z, s);
              s = fmaf(av[c].w, xv.w, s);
              d[c * K + v] = s;
            }
          }
        }
        const float red = team_allreduce<NV>(d, part, buf, warp, lane, P, team, team_warp0);
        // the NV totals to every lane through this warp's shared-memory slot: one store and
        // broadcast loads instead of NV shuffles (measured on the B200: 7 % off the batch)
        float* bcw = bcast + warp * 32;
        __syncwarp();
        if ((lane % (32 / NV)) == 0) bcw[lane / (32 / NV)] = red;
        __syncwarp();
        if constexpr (K % 2 == 0) {
#pragma unroll
          for (int c = 0; c < GC; ++c)
#pragma unroll
            for (int vp = 0; vp < K / 2; ++vp) {
              float2 tc = *reinterpret_cast<const float2*>(bcw + c * K + 2 * vp);
              if (wamm) tc = __fmul2_rn(tc, make_float2(wt[c], wt[c]));
              const float ae[4] = {av[c].x, av[c].y, av[c].z, av[c].w};
#pragma unroll
              for (int e = 0; e < 4; ++e) {
                const float2 y2 = __ffma2_rn(make_float2(ae[e], ae[e]), tc,
                                             make_float2(Y[e][2 * vp], Y[e][2 * vp + 1]));
                Y[e][2 * vp] = y2.x;
                Y[e][2 * vp + 1] = y2.y;
              }
            }
        } else {
#pragma unroll
          for (int c = 0; c < GC; ++c)
#pragma unroll
            for (int v = 0; v < K; ++v) {
              const float tc = bcw[c * K + v] * wt[c];
              Y[0][v] = fmaf(av[c].x, tc, Y[0][v]);
              Y[1][v] = fmaf(av[c].y, tc, Y[1][v]);
              Y[2][v] = fmaf(av[c].z, tc, Y[2][v]);
              Y[3][v] = fmaf(av[c].w, tc, Y[3][v]);
            }
        }
      };
      // rows past m (the padding up to ld) are zero-filled, so are the slots past the list
      const int gstep = NTG * GC;
      constexpr int NST = Ring<GC>::stages;
      static_assert(NST >= 3, "the column ring needs at least 3 stages");
      // the ring: NST - 1 groups in flight while one is multiplied
      float4* ring = reinterpret_cast<float4*>(smem + SL::region);
      const int vbytes = rows ? 4 * min(4, m - r0) : 0;
      auto issue = [&](int g0, int slot) {
#pragma unroll
        for (int c = 0; c < GC; ++c) {
          const int col = (g0 + c < ncols) ? (wamm ? lcol[g0 + c] : g0 + c) : -1;
          const bool live = vbytes > 0 && col >= 0;
          cp_async16_zfill(ring + (slot * GC + c) * kThreads + t,
                           live ? Ab + (int64_t)col * M.ld : M.A, live ? vbytes : 0);
        }
      };
      int gi = gteam * GC;  // next group to copy
#pragma unroll 1
      for (int s = 0; s < NST - 1; ++s, gi += gstep) {
        if (gi < ncols) issue(gi, s);
        cp_async_commit();
      }
      int slot = 0;
#pragma unroll 1
      for (int g0 = gteam * GC; g0 < ncols; g0 += gstep, buf ^= 1) {
        cp_async_wait_group<NST - 2>();  // group g0 has landed (this thread's copies)
        // refill the slot this thread emptied in the previous group
        if (gi < ncols) issue(gi, slot == 0 ? NST - 1 : slot - 1);
        cp_async_commit();
        gi += gstep;
        float4 av[GC];
        float wt[GC];
#pragma unroll
        for (int c = 0; c < GC; ++c) {
          av[c] = lds_f4(reinterpret_cast<const float*>(ring + (slot * GC + c) * kThreads + t));
          wt[c] = (wamm && g0 + c < ncols) ? lw[g0 + c] : 1.f;
        }
        multiply(av, wt);
        slot = (slot + 1 == NST) ? 0 : slot + 1;
      }
      cp_async_wait_all();  // only empty groups can still be open here
      }
      // ---- sum the team partials of Y (fixed order), every team receives the total ----
      if (!TC && NT > 1) {
        __syncthreads();
        if (rows) {
#pragma unroll
          for (int e = 0; e < 4; ++e)
#pragma unroll
            for (int v = 0; v < K; ++v) yred[((team * 4 * P) + r0 + e) * K + v] = Y[e][v];
        }
        __syncthreads();
        if (rows && team == 0) {  // only team 0 uses the summed Y (Gram, residual, X, v)
#pragma unroll
          for (int e = 0; e < 4; ++e)
#pragma unroll
            for (int v = 0; v < K; ++v) {
              float s = 0.f;
              for (int tm = 0; tm < NT; ++tm) s += yred[((tm * 4 * P) + r0 + e) * K + v];
              Y[e][v] = s;
            }
        }
      }
      // ---- sum the CTA partials of the cluster through distributed shared memory (fixed
      // rank order): every CTA receives the same Y ----
      if (CL > 1) {
        __syncthreads();
        if (team == 0 && rows) {
#pragma unroll
          for (int e = 0; e < 4; ++e)
#pragma unroll
            for (int v = 0; v < K; ++v) yred[(r0 + e) * K + v] = Y[e][v];
        }
        cluster.sync();
        if (rows && team == 0) {
#pragma unroll
          for (int e = 0; e < 4; ++e)
#pragma unroll
            for (int v = 0; v < K; ++v) {
              float s = 0.f;
              for (int rk = 0; rk < CL; ++rk)
                s += *cluster.map_shared_rank(&yred[(r0 + e) * K + v], rk);
              Y[e][v] = s;
            }
        }
        cluster.sync();  // the buffers are rewritten by the next step
      }
      // ---- variance reduction: Y = Y_memo·S + Ĉ·D for a sampled product; an exact product
      // becomes the memo pair (team 0, its own rows, in every CTA of the cluster alike) ----
      if (use_d) {
        // no team reads X or D any more: every team passed a barrier after its product pass
        // (team sums, cluster sums) or team 0 is the only team
        if (team == 0) vr_add_memo<K>(Y, Ym, Svr, Xsave, Xs, r0);
      }
      if (vr && exact_p) {
        if (team == 0) vr_store_memo<K>(Y, Xm, Ym, Xs, r0);
        memo = true;
      }
      prev_exact = exact_p;
    }
    __syncthreads();
  }
}

// ---- backward: grad_b = 2·v_b·(v_bᵀ·A_b), column-major like A_b, one warp per column ----
struct GradArgs {
  const Mat* mats;
  const int64_t* col_start;  // count + 1 prefix of column counts
  int32_t count;
  const float* vec;          // Σ m
  float* const* grads;       // count pointers
  const int64_t* grad_ld;    // count
  const float* scale;        // count (upstream gradient per matrix), or null (1)
  int32_t vs_len;            // floats of a warp's copy of v: the largest m, rounded up to 4
};

// Column prefixes a CTA of the backward keeps in shared memory (larger batches search global
// memory).
constexpr int kGradSmemMats = 4096;

// Each warp takes a contiguous range of columns (an even share of all the batch's columns), two
// adjacent columns at a time: both columns' loads are in flight together and their two dots
// share one warp reduction.  The matrix of a column is found in the column prefix (copied to
// shared memory once per CTA) by a search forward from the warp's previous matrix; when the warp
// enters a matrix it copies v into its own 16-byte aligned shared-memory slot, so that A, v and
// the gradient all move in 16-byte accesses (A and the gradient streaming; a gradient column
// that does not start 16-byte aligned takes 4-byte stores).
struct GradMat {
  Mat M;
  int64_t c0 = 0, c1 = 0;  // column range
  float* g = nullptr;
  int64_t gld = 0;
  float k = 1.f;  // 2·scale
  int mi = -1;
};

__device__ __forceinline__ void grad_store(const GradMat& G, const float* vs, int64_t j, float k,
                                           int lane) {
  const int m = G.M.m, m4 = m >> 2;
  float* g = G.g + j * G.gld;
  if ((reinterpret_cast<uintptr_t>(g) & 15u) == 0u) {
#pragma unroll 4
    for (int r4 = lane; r4 < m4; r4 += 32) {
      const float4 vv = reinterpret_cast<const float4*>(vs)[r4];
      __stcs(reinterpret_cast<float4*>(g) + r4, make_float4(k * vv.x, k * vv.y, k * vv.z, k * vv.w));
    }
    for (int r = 4 * m4 + lane; r < m; r += 32) g[r] = k * vs[r];
  } else {
    for (int r = lane; r < m; r += 32) g[r] = k * vs[r];
  }
}

// this lane's part of the dot of column j with v
__device__ __forceinline__ float grad_dot(const GradMat& G, const float* vs, int64_t j, int lane) {
  const int m = G.M.m, m4 = m >> 2;
  const float4* col4 = reinterpret_cast<const float4*>(G.M.A + j * G.M.ld);
  float s = 0.f;
#pragma unroll 4
  for (int r4 = lane; r4 < m4; r4 += 32) {
    const float4 c = __ldcs(col4 + r4);
    const float4 vv = reinterpret_cast<const float4*>(vs)[r4];
    s = fmaf(c.x, vv.x, s);
    s = fmaf(c.y, vv.y, s);
    s = fmaf(c.z, vv.z, s);
    s = fmaf(c.w, vv.w, s);
  }
  for (int r = 4 * m4 + lane; r < m; r += 32) s = fmaf(G.M.A[j * G.M.ld + r], vs[r], s);
  return s;
}

__global__ void __launch_bounds__(256, 4) grad_kernel(const __grid_constant__ GradArgs a) {
  // dynamic shared memory: 8 warp slots of vs_len floats (16-byte multiples), then the column
  // prefixes when count <= kGradSmemMats
  extern __shared__ __align__(16) unsigned char gsm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float* vs = reinterpret_cast<float*>(gsm) + (size_t)warp * a.vs_len;
  int64_t* cs_s = reinterpret_cast<int64_t*>(gsm + sizeof(float) * 8 * (size_t)a.vs_len);
  const int count = a.count;
  const bool in_smem = count <= kGradSmemMats;
  if (in_smem)
    for (int i = threadIdx.x; i <= count; i += blockDim.x) cs_s[i] = a.col_start[i];
  __syncthreads();
  auto cstart = [&](int i) -> int64_t { return in_smem ? cs_s[i] : __ldg(a.col_start + i); };
  // the matrix holding column gc (gc not below the range of G): forward search from G's; on a
  // change v is copied into this warp's slot (every lane reads only after the __syncwarp)
  auto locate = [&](GradMat& G, int64_t gc) {
    if (gc < G.c1) return;
    int lo = G.mi + 1, hi = count - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (cstart(mid) <= gc)
        lo = mid;
      else
        hi = mid - 1;
    }
    G.mi = lo;
    G.M = a.mats[lo];
    G.c0 = cstart(lo);
    G.c1 = cstart(lo + 1);
    G.g = a.grads[lo];
    G.gld = a.grad_ld[lo];
    G.k = 2.f * (a.scale ? a.scale[lo] : 1.f);
    __syncwarp();  // every lane is done with the slot's previous vector
    const float* v = a.vec + G.M.out_off;
    for (int r = lane; r < G.M.m; r += 32) vs[r] = v[r];
    __syncwarp();
  };
  const int64_t total = cstart(count);
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t b0 = gw * total / nw, b1 = (gw + 1) * total / nw;  // this warp's columns
  GradMat G;
  for (int64_t gc = b0; gc < b1;) {
    locate(G, gc);
    const int64_t j = gc - G.c0;
    if (gc + 1 < b1 && gc + 1 < G.c1) {  // two columns of one matrix (the usual case)
      float d[2] = {grad_dot(G, vs, j, lane), grad_dot(G, vs, j + 1, lane)};
      const float s = warp_reduce_multi<float, 2>(d, lane);  // lane < 16: column j, else j + 1
      const float s0 = __shfl_sync(0xffffffffu, s, 0), s1 = __shfl_sync(0xffffffffu, s, 16);
      grad_store(G, vs, j, G.k * s0, lane);
      grad_store(G, vs, j + 1, G.k * s1, lane);
      gc += 2;
    } else {
      const float s0 = warp_sum(grad_dot(G, vs, j, lane));
      grad_store(G, vs, j, G.k * s0, lane);
      gc += 1;
    }
  }
}

using KernelFn = void (*)(Args);

struct Variant {
  int K, GC;
  KernelFn fn;
  bool tc;  // tensor-core product: exact batches only
};
constexpr int kClusterSizes[] = {1, 2, 4, 8};

static const Variant kVariants[] = {
    {1, 2, batch_kernel<1, 2>, false},
    {1, 4, batch_kernel<1, 4>, false},
    {4, 2, batch_kernel<4, 2>, false},
    {4, 4, batch_kernel<4, 4>, false},
    {8, 1, batch_kernel<8, 1>, false},
    {8, 2, batch_kernel<8, 2>, false},
    {8, 4, batch_kernel<8, 4>, false},
    {8, kTcCols, batch_kernel<8, kTcCols, true>, true},
};

static int smem_bytes(const Variant& V, bool amm) {
  if (V.tc) return Smem<8, true>::total;
  switch (V.K) {
    case 1: return amm ? Smem<1>::total_amm : Smem<1>::total;
    case 4: return amm ? Smem<4>::total_amm : Smem<4>::total;
    default: return amm ? Smem<8>::total_amm : Smem<8>::total;
  }
}

}  // namespace batch
}  // namespace amm

// ------------------------------------------------------------------------------------------
// Host side: the batch context
// ------------------------------------------------------------------------------------------
using amm::batch::Mat;

struct amm_batch {
  int device = 0;
  int nsm = 0;
  amm_batch_config cfg{};
  int64_t count = 0;
  std::vector<Mat> mats;
  std::vector<int32_t> order;
  int64_t vec_len = 0;
  int64_t total_cols = 0;
  int64_t n_states = 0;
  bool amm = false;
  // device memory (one allocation)
  void* mem = nullptr;
  Mat* d_mats = nullptr;
  int32_t* d_order = nullptr;
  uint32_t* d_queue = nullptr;
  int64_t* d_col_start = nullptr;
  float** d_grads = nullptr;
  int64_t* d_grad_ld = nullptr;
  uint32_t* d_states0 = nullptr;  // seeded xorshift states (AMM mode), copied per run
  uint32_t* d_states = nullptr;
  float* d_vr = nullptr;          // AMM mode with variance reduction: per-CTA memo pairs
  // exact batches of 8 vectors: one tensor map per matrix for the tensor-core kernel's tile
  // copies (null when they cannot be encoded; that kernel is then not a candidate)
  CUtensorMap* d_tmaps = nullptr;
  std::vector<CUtensorMap> h_tmaps;
  // optional record of the CDFs and picks (amm_batch_record)
  float* rec_cdf = nullptr;
  uint32_t* rec_picks = nullptr;
  int rec_products = 0;
  int variant = -1;  // chosen tile shape (index into kVariants)
  int cluster = 1;   // CTAs per matrix (cluster size)
  int grid = 0;      // CTAs of the persistent launch for that cluster size
  // The heaviest matrices on a wide-cluster launch (wide_count 0: one launch per run): it takes
  // the first wide_count matrices of the order on clusters of wide_cluster CTAs, then joins
  // the launch queued behind it (clusters of `cluster`, narrow_grid CTAs) on the rest.
  int wide_count = 0;
  int wide_cluster = 0;
  int wide_grid = 0;
  int narrow_grid = 0;
  float wide_ms = 0.f;   // the plan's time in the autotuner (0: not timed)
  std::map<std::pair<int, int>, float> tune_ms;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  cudaStream_t cap = nullptr;
  double* g_lam = nullptr;
  float* g_vec = nullptr;
  int32_t* g_iters = nullptr;
};

namespace {

int fail(cudaError_t e, const char* what) { return amm::record_cuda_failure(e, what); }

#define BATCH_CUDA(call)                            \
  do {                                              \
    cudaError_t e_ = (call);                        \
    if (e_ != cudaSuccess) return fail(e_, #call);  \
  } while (0)

struct Guard {
  int old = -1;
  explicit Guard(int dev) {
    cudaGetDevice(&old);
    if (old != dev) cudaSetDevice(dev);
  }
  ~Guard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (old >= 0 && cur != old) cudaSetDevice(old);
  }
};

// Clusters of cl CTAs of the given tile shape that are resident at once (one CTA per SM); 0 if
// that cluster size cannot run.
int max_clusters(amm_batch* b, int variant, int cl) {
  const auto& V = amm::batch::kVariants[variant];
  const int sm = amm::batch::smem_bytes(V, b->amm);
  if (cudaFuncSetAttribute(V.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, sm) != cudaSuccess)
    return 0;
  if (cl > 1 &&
      cudaFuncSetAttribute(V.fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)
    return 0;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(cl * b->nsm, 1, 1);
  cfg.blockDim = dim3(amm::batch::kThreads, 1, 1);
  cfg.dynamicSmemBytes = sm;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = cl;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  int nclusters = 0;
  if (cudaOccupancyMaxActiveClusters(&nclusters, (void*)V.fn, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return nclusters > 0 ? nclusters : 0;
}

// CTAs of a persistent launch with clusters of cl CTAs: as many clusters as fit at once, and
// no more than there are matrices.  0 if that cluster size cannot run.
int persistent_grid(amm_batch* b, int variant, int cl) {
  const int nclusters = max_clusters(b, variant, cl);
  if (nclusters < 1) return 0;
  const int64_t use = std::min<int64_t>(nclusters, b->count);
  return (int)use * cl;
}

// Start of a run: both work-list counters zeroed and, in AMM mode, the seeded states restored
// (every run draws the same picks).
int run_prologue(amm_batch* b, cudaStream_t s) {
  BATCH_CUDA(cudaMemsetAsync(b->d_queue, 0, 2 * sizeof(uint32_t), s));
  if (b->amm)
    BATCH_CUDA(cudaMemcpyAsync(b->d_states, b->d_states0, sizeof(uint32_t) * b->n_states,
                               cudaMemcpyDeviceToDevice, s));
  return AMM_OK;
}

// One persistent launch over the shared list (order, count), after its own list (order0,
// count0).  dependent: launched as a programmatic dependent of the launch before it in the
// stream, so that it starts on the SMs that launch leaves free.
int launch_kernel(amm_batch* b, int variant, int cl, int grid, double* d_lam, float* d_vec,
                  int32_t* d_iters, int max_iter, const int32_t* order, int count,
                  const int32_t* order0, int count0, bool dependent, cudaStream_t s,
                  int vr_base = 0) {
  const auto& V = amm::batch::kVariants[variant];
  const int sm = amm::batch::smem_bytes(V, b->amm);
  BATCH_CUDA(cudaFuncSetAttribute(V.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
  if (cl > 1)
    BATCH_CUDA(cudaFuncSetAttribute(V.fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  amm::batch::Args a{};
  a.mats = b->d_mats;
  a.order = order;
  a.count = count;
  a.order0 = order0;
  a.count0 = count0;
  a.max_iter = max_iter;
  a.tol = b->cfg.tol;
  a.rr_period = b->cfg.rr_period > 0 ? b->cfg.rr_period : 1;
  a.seed = b->cfg.seed;
  a.queue = b->d_queue;
  a.states = b->d_states;
  a.lam = d_lam;
  a.vec = d_vec;
  a.iters = d_iters;
  a.vr_period = b->d_vr ? b->cfg.vr_period : 0;
  a.vr_base = vr_base;
  a.vr_mem = b->d_vr;
  a.rec_cdf = b->rec_cdf;
  a.rec_picks = b->rec_picks;
  a.rec_products = b->rec_products;
  a.col_start = b->d_col_start;
  a.tmaps = b->d_tmaps;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid, 1, 1);
  cfg.blockDim = dim3(amm::batch::kThreads, 1, 1);
  cfg.dynamicSmemBytes = sm;
  cfg.stream = s;
  cudaLaunchAttribute at[2];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = cl;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[1].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = dependent ? 2 : 1;
  BATCH_CUDA(cudaLaunchKernelEx(&cfg, V.fn, a));
  amm::count_launch(1);
  BATCH_CUDA(cudaGetLastError());
  return AMM_OK;
}

// A run as one launch over the order list (or a slice of it).
int launch(amm_batch* b, int variant, int cl, int grid, double* d_lam, float* d_vec,
           int32_t* d_iters, int max_iter, const int32_t* order, int count, cudaStream_t s) {
  const int rc = run_prologue(b, s);
  if (rc) return rc;
  return launch_kernel(b, variant, cl, grid, d_lam, d_vec, d_iters, max_iter, order, count,
                       nullptr, 0, false, s);
}

// A run with the wide-cluster plan: the wide launch takes the heaviest matrices first, the
// launch queued behind it (programmatic dependent) takes the SMs left, and both share the rest
// of the order list.
int launch_wide(amm_batch* b, double* d_lam, float* d_vec, int32_t* d_iters, int max_iter,
                cudaStream_t s) {
  int rc = run_prologue(b, s);
  if (rc) return rc;
  const int32_t* rest = b->d_order + b->wide_count;
  const int nrest = (int)b->count - b->wide_count;
  rc = launch_kernel(b, b->variant, b->wide_cluster, b->wide_grid, d_lam, d_vec, d_iters,
                     max_iter, rest, nrest, b->d_order, b->wide_count, false, s);
  if (rc) return rc;
  return launch_kernel(b, b->variant, b->cluster, b->narrow_grid, d_lam, d_vec, d_iters,
                       max_iter, rest, nrest, nullptr, 0, true, s, b->wide_grid);
}

// The run of the chosen plan.
int launch_run(amm_batch* b, double* d_lam, float* d_vec, int32_t* d_iters, cudaStream_t s) {
  if (b->wide_count > 0) return launch_wide(b, d_lam, d_vec, d_iters, (int)b->cfg.max_iter, s);
  return launch(b, b->variant, b->cluster, b->grid, d_lam, d_vec, d_iters,
                (int)b->cfg.max_iter, b->d_order, (int)b->count, s);
}

// Wide-cluster plan for a batch of uneven matrices.  With one cluster size for all, a matrix
// whose work alone, on one cluster, exceeds an even share of the whole batch per cluster sets
// the run's time (the queue hands it out first, but nothing can help with it).  Those leading
// matrices of the order go to a launch with clusters large enough for the heaviest (the next
// sizes up, at most 8) on at most half the SMs; it then helps with the rest.  Needs
// programmatic dependent launch (both launches resident at once).  With the default setting
// (wide = 0) only for an autotuned cluster size; wide = 1 plans it for a fixed one too, and
// wide = -1 never.
void plan_wide(amm_batch* b) {
  b->wide_count = 0;
  if (!amm::pdl_enabled() || b->cfg.wide < 0 || b->count < 2) return;
  if (b->cfg.cluster > 0 && b->cfg.wide == 0) return;
  double total = 0.0;
  for (const Mat& x : b->mats) total += (double)x.m * (double)x.n;
  // work per SM of an even split, with a margin: the per-CTA rate falls with the row count,
  // so the heaviest matrices are also the slowest per element
  const double share = 0.75 * total / (double)b->nsm;
  auto work = [&](int k) { const Mat& x = b->mats[b->order[k]]; return (double)x.m * x.n; };
  int nwide = 0;
  while (nwide < b->count && work(nwide) > (double)b->cluster * share) ++nwide;
  if (nwide == 0) return;
  int wcl = 0;
  for (int cl : amm::batch::kClusterSizes) {
    if (cl <= b->cluster) continue;
    wcl = cl;
    if (work(0) <= (double)cl * share) break;
  }
  if (wcl == 0) return;
  int nclusters = std::min(max_clusters(b, b->variant, wcl), (b->nsm / 2) / wcl);
  nclusters = std::min(nclusters, nwide);
  if (nclusters < 1) return;
  const int wide_grid = nclusters * wcl;
  int narrow = (b->nsm - wide_grid) / b->cluster;
  narrow = std::min(narrow, max_clusters(b, b->variant, b->cluster));
  narrow = (int)std::min<int64_t>(narrow, b->count - nwide);
  if (narrow < 1) return;
  b->wide_count = nwide;
  b->wide_cluster = wcl;
  b->wide_grid = wide_grid;
  b->narrow_grid = narrow * b->cluster;
}

// Tile-shape autotuner: every (columns per group, cluster size) pair with the requested K runs
// the whole batch for up to 20 iterations (enough for the per-matrix set-up, which favours
// larger clusters, to weigh as it does in a real run); the fastest of two timed runs (CUDA
// events) is kept for the context.
int autotune(amm_batch* b, double* d_lam, float* d_vec, int32_t* d_iters, cudaStream_t s) {
  if (b->variant >= 0) return AMM_OK;
  int best = -1, best_cl = 1, best_grid = 0;
  float best_ms = 0.f;
  cudaEvent_t e0, e1;
  BATCH_CUDA(cudaEventCreate(&e0));
  BATCH_CUDA(cudaEventCreate(&e1));
  const int n_var = (int)(sizeof(amm::batch::kVariants) / sizeof(amm::batch::kVariants[0]));
  // the candidates; a single one (tile and cluster size fixed by the caller) is taken untimed
  std::vector<std::tuple<int, int, int>> cand;  // (variant, cluster size, grid)
  for (int v = 0; v < n_var; ++v) {
    if (amm::batch::kVariants[v].K != b->cfg.nvec) continue;
    if (amm::batch::kVariants[v].tc && (b->amm || !b->d_tmaps)) continue;  // exact-only, maps
    if (b->cfg.tile_gc > 0 && amm::batch::kVariants[v].GC != b->cfg.tile_gc) continue;
    for (int cl : amm::batch::kClusterSizes) {
      if (b->cfg.cluster > 0 && cl != b->cfg.cluster) continue;
      const int grid = persistent_grid(b, v, cl);
      if (grid > 0) cand.emplace_back(v, cl, grid);
    }
  }
  if (cand.size() == 1) {
    b->variant = std::get<0>(cand[0]);
    b->cluster = std::get<1>(cand[0]);
    b->grid = std::get<2>(cand[0]);
    plan_wide(b);  // only with wide = 1 (the cluster size is the caller's); untimed
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return AMM_OK;
  }
  for (const auto& cd : cand) {
    const int v = std::get<0>(cd), cl = std::get<1>(cd), grid = std::get<2>(cd);
    const int iters = (int)std::min<int64_t>(b->cfg.max_iter, 20);
    int rc = launch(b, v, cl, grid, d_lam, d_vec, d_iters, iters, b->d_order, (int)b->count, s);
    if (rc) return rc;
    float ms = 0.f;
    for (int rep = 0; rep < 2; ++rep) {
      BATCH_CUDA(cudaEventRecord(e0, s));
      rc = launch(b, v, cl, grid, d_lam, d_vec, d_iters, iters, b->d_order, (int)b->count, s);
      if (rc) return rc;
      BATCH_CUDA(cudaEventRecord(e1, s));
      BATCH_CUDA(cudaEventSynchronize(e1));
      float t = 0.f;
      BATCH_CUDA(cudaEventElapsedTime(&t, e0, e1));
      ms = rep == 0 ? t : std::min(ms, t);
    }
    b->tune_ms[{v, cl}] = ms;
    if (best < 0 || ms < best_ms) {
      best = v;
      best_cl = cl;
      best_grid = grid;
      best_ms = ms;
    }
  }
  if (best < 0) {
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return AMM_ERR_UNSUPPORTED;
  }
  b->variant = best;
  b->cluster = best_cl;
  b->grid = best_grid;
  // the wide-cluster plan, kept only if it runs faster (same iterations, best of two), or
  // untimed with wide = 1
  plan_wide(b);
  if (b->wide_count > 0 && b->cfg.wide == 0) {
    const int iters = (int)std::min<int64_t>(b->cfg.max_iter, 20);
    int rc = launch_wide(b, d_lam, d_vec, d_iters, iters, s);
    float ms = 0.f;
    for (int rep = 0; rc == AMM_OK && rep < 2; ++rep) {
      BATCH_CUDA(cudaEventRecord(e0, s));
      rc = launch_wide(b, d_lam, d_vec, d_iters, iters, s);
      if (rc) break;
      BATCH_CUDA(cudaEventRecord(e1, s));
      BATCH_CUDA(cudaEventSynchronize(e1));
      float t = 0.f;
      BATCH_CUDA(cudaEventElapsedTime(&t, e0, e1));
      ms = rep == 0 ? t : std::min(ms, t);
    }
    b->wide_ms = ms;
    if (rc || !(ms < best_ms)) b->wide_count = 0;
    if (rc) {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      return rc;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return AMM_OK;
}

}  // namespace

extern "C" {

void amm_batch_config_default(amm_batch_config* c) {
  if (!c) return;
  std::memset(c, 0, sizeof(*c));
  c->nvec = 8;
  c->max_iter = 500;
  c->tol = 1e-6;
  c->rr_period = 1;
  c->use_graph = 1;
  c->seed = 1234;
  c->tile_gc = 0;
  c->c_divisor = 0;
  c->cluster = 0;
  c->wide = 0;
  c->vr_period = 0;
}

// The driver's tensor-map encoder (cuTensorMapEncodeTiled), looked up once through the
// runtime; null if the driver does not offer it.
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}

// The tensor maps of the tensor-core kernel's tile copies, one per matrix: FP32, dims {m, n}
// (rows innermost; row stride ld·4 bytes, a multiple of 16 by the batch's alignment rule),
// boxes of 32 rows x 8 columns with the 128-byte swizzle, zeros outside the matrix.  False if
// any cannot be encoded.
static bool encode_tensor_maps(const std::vector<Mat>& ms, std::vector<CUtensorMap>& out) {
  const auto enc = tensor_map_encoder();
  if (!enc) return false;
  out.resize(ms.size());
  for (size_t i = 0; i < ms.size(); ++i) {
    const Mat& M = ms[i];
    const cuuint64_t dims[2] = {(cuuint64_t)M.m, (cuuint64_t)M.n};
    const cuuint64_t strides[1] = {(cuuint64_t)M.ld * sizeof(float)};
    const cuuint32_t box[2] = {32, (cuuint32_t)amm::batch::kTcCols};
    const cuuint32_t elem[2] = {1, 1};
    if (enc(&out[i], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(M.A), dims, strides,
            box, elem, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
            CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return false;
  }
  return true;
}

int amm_batch_create(amm_batch** out, const amm_batch_matrix* mats, int64_t count,
                     const amm_batch_config* cfg, int device) {
  if (!out || !mats || !cfg || count < 1 || count > (1 << 20)) return AMM_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (cfg->nvec != 1 && cfg->nvec != 4 && cfg->nvec != 8) return AMM_ERR_UNSUPPORTED;
  if (cfg->max_iter < 1 || !(cfg->tol >= 0.0) || cfg->rr_period < 0 || cfg->c_divisor < 0 ||
      cfg->wide < -1 || cfg->wide > 1 || cfg->vr_period < 0)
    return AMM_ERR_INVALID_ARGUMENT;
  const bool amm_mode = cfg->c_divisor > 0;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return AMM_ERR_NO_DEVICE;
  if (device < 0 || device >= ndev) return AMM_ERR_INVALID_ARGUMENT;
  std::vector<Mat> ms((size_t)count);
  int64_t off = 0, cols = 0, nst = 0;
  for (int64_t i = 0; i < count; ++i) {
    const amm_batch_matrix& x = mats[i];
    if (!x.A || x.m < 1 || x.n < 1 || x.ld < x.m) return AMM_ERR_INVALID_ARGUMENT;
    if (x.m > amm::batch::kMaxRows || x.n > INT32_MAX) return AMM_ERR_UNSUPPORTED;
    if (x.m < cfg->nvec) return AMM_ERR_UNSUPPORTED;
    if ((reinterpret_cast<uintptr_t>(x.A) & 15) != 0 || (x.ld % 4) != 0) return AMM_ERR_ALIGNMENT;
    ms[i].A = static_cast<const float*>(x.A);
    ms[i].ld = x.ld;
    ms[i].m = (int32_t)x.m;
    ms[i].n = (int32_t)x.n;
    ms[i].out_off = off;
    ms[i].st_off = nst;
    ms[i].c = 0;
    if (amm_mode) {
      if (x.n > amm::batch::kMaxCols) return AMM_ERR_UNSUPPORTED;
      int64_t c = x.n / cfg->c_divisor;
      if (c < 1) c = 1;
      if (c > amm::batch::kMaxPicks) return AMM_ERR_UNSUPPORTED;
      ms[i].c = (int32_t)c;
      nst += c;
    }
    off += x.m;
    cols += x.n;
  }
  amm_batch* b = new amm_batch();
  b->device = device;
  b->cfg = *cfg;
  b->count = count;
  b->mats = ms;
  b->vec_len = off;
  b->total_cols = cols;
  b->n_states = nst;
  b->amm = amm_mode;
  b->order.resize((size_t)count);
  for (int64_t i = 0; i < count; ++i) b->order[i] = (int32_t)i;
  // largest first (work m·n), ties by index: the queue then balances like LPT scheduling
  std::stable_sort(b->order.begin(), b->order.end(), [&](int32_t x, int32_t y) {
    return (int64_t)ms[x].m * ms[x].n > (int64_t)ms[y].m * ms[y].n;
  });
  Guard g(device);
  cudaDeviceGetAttribute(&b->nsm, cudaDevAttrMultiProcessorCount, device);
  size_t bytes = 0;
  auto carve = [&](size_t n, size_t align) {
    bytes = (bytes + align - 1) / align * align;
    const size_t o = bytes;
    bytes += n;
    return o;
  };
  const size_t o_mats = carve(sizeof(Mat) * count, 256);
  const size_t o_order = carve(sizeof(int32_t) * count, 256);
  const size_t o_queue = carve(sizeof(uint32_t) * 4, 256);
  const size_t o_cols = carve(sizeof(int64_t) * (count + 1), 256);
  const size_t o_grads = carve(sizeof(float*) * count, 256);
  const size_t o_gld = carve(sizeof(int64_t) * count, 256);
  const size_t o_st0 = carve(sizeof(uint32_t) * (nst > 0 ? nst : 1), 256);
  const size_t o_st = carve(sizeof(uint32_t) * (nst > 0 ? nst : 1), 256);
  // memo pairs of the variance reduction: one slot per CTA that can be resident at once (the
  // launches of a run hold at most one CTA per SM between them)
  const bool with_vr = amm_mode && cfg->vr_period > 0;
  const size_t vr_floats = (size_t)amm::batch::kVrSlot * amm::batch::kMaxRows * cfg->nvec;
  const size_t o_vr = with_vr ? carve(sizeof(float) * vr_floats * b->nsm, 256) : 0;
  // tensor maps (64-byte aligned each) when the tensor-core kernel can run: exact, 8 vectors
  const bool with_tmaps = !amm_mode && cfg->nvec == 8 && encode_tensor_maps(ms, b->h_tmaps);
  const size_t o_tmaps = with_tmaps ? carve(sizeof(CUtensorMap) * count, 256) : 0;
  cudaError_t e = cudaMalloc(&b->mem, bytes);
  if (e != cudaSuccess) {
    delete b;
    return e == cudaErrorMemoryAllocation ? AMM_ERR_OUT_OF_MEMORY : fail(e, "cudaMalloc");
  }
  char* base = static_cast<char*>(b->mem);
  b->d_mats = reinterpret_cast<Mat*>(base + o_mats);
  b->d_order = reinterpret_cast<int32_t*>(base + o_order);
  b->d_queue = reinterpret_cast<uint32_t*>(base + o_queue);
  b->d_col_start = reinterpret_cast<int64_t*>(base + o_cols);
  b->d_grads = reinterpret_cast<float**>(base + o_grads);
  b->d_grad_ld = reinterpret_cast<int64_t*>(base + o_gld);
  b->d_states0 = reinterpret_cast<uint32_t*>(base + o_st0);
  b->d_states = reinterpret_cast<uint32_t*>(base + o_st);
  b->d_vr = with_vr ? reinterpret_cast<float*>(base + o_vr) : nullptr;
  b->d_tmaps = with_tmaps ? reinterpret_cast<CUtensorMap*>(base + o_tmaps) : nullptr;
  std::vector<int64_t> cs((size_t)count + 1, 0);
  for (int64_t i = 0; i < count; ++i) cs[i + 1] = cs[i] + ms[i].n;
  e = cudaMemcpy(b->d_mats, ms.data(), sizeof(Mat) * count, cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(b->d_order, b->order.data(), sizeof(int32_t) * count, cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(b->d_col_start, cs.data(), sizeof(int64_t) * (count + 1),
                   cudaMemcpyHostToDevice);
  if (e == cudaSuccess && with_tmaps)
    e = cudaMemcpy(b->d_tmaps, b->h_tmaps.data(), sizeof(CUtensorMap) * count,
                   cudaMemcpyHostToDevice);
  if (e == cudaSuccess && nst > 0) {
    // xorshift32 states: a splitmix64 stream from the seed (never zero, a fixed point)
    std::vector<uint32_t> st((size_t)nst);
    uint64_t z = cfg->seed;
    for (int64_t k = 0; k < nst; ++k) {
      z += 0x9E3779B97F4A7C15ull;
      uint64_t x = z;
      x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
      x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
      x ^= x >> 31;
      const uint32_t v = (uint32_t)(x >> 32);
      st[(size_t)k] = v ? v : 0x6A09E667u;
    }
    e = cudaMemcpy(b->d_states0, st.data(), sizeof(uint32_t) * nst, cudaMemcpyHostToDevice);
  }
  if (e != cudaSuccess) {
    cudaFree(b->mem);
    delete b;
    return fail(e, "cudaMemcpy(batch descriptors)");
  }
  *out = b;
  return AMM_OK;
}

int amm_batch_destroy(amm_batch* b) {
  if (!b) return AMM_ERR_INVALID_ARGUMENT;
  Guard g(b->device);
  if (b->gexec) cudaGraphExecDestroy(b->gexec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->cap) cudaStreamDestroy(b->cap);
  if (b->mem) cudaFree(b->mem);
  delete b;
  return AMM_OK;
}

int amm_batch_vector_offsets(amm_batch* b, int64_t* offsets) {
  if (!b || !offsets) return AMM_ERR_INVALID_ARGUMENT;
  for (int64_t i = 0; i < b->count; ++i) offsets[i] = b->mats[i].out_off;
  offsets[b->count] = b->vec_len;
  return AMM_OK;
}

int amm_batch_run(amm_batch* b, double* d_lambda, float* d_vectors, int32_t* d_iters,
                  void* stream) {
  if (!b || !d_lambda || !d_vectors || !d_iters) return AMM_ERR_INVALID_ARGUMENT;
  Guard g(b->device);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  int rc = autotune(b, d_lambda, d_vectors, d_iters, s);
  if (rc) return rc;
  if (!b->cfg.use_graph) return launch_run(b, d_lambda, d_vectors, d_iters, s);
  if (b->gexec && (b->g_lam != d_lambda || b->g_vec != d_vectors || b->g_iters != d_iters)) {
    cudaGraphExecDestroy(b->gexec);
    cudaGraphDestroy(b->graph);
    b->gexec = nullptr;
    b->graph = nullptr;
  }
  if (!b->gexec) {
    if (!b->cap) BATCH_CUDA(cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking));
    BATCH_CUDA(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeRelaxed));
    const int64_t before = amm::launch_count();
    rc = launch_run(b, d_lambda, d_vectors, d_iters, b->cap);
    cudaGraph_t gr = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(b->cap, &gr);
    amm::count_launch(-(int)(amm::launch_count() - before));
    if (rc) {
      if (gr) cudaGraphDestroy(gr);
      return rc;
    }
    if (ce != cudaSuccess) return fail(ce, "cudaStreamEndCapture");
    const cudaError_t ie = cudaGraphInstantiate(&b->gexec, gr, 0);
    if (ie != cudaSuccess) {
      cudaGraphDestroy(gr);
      return fail(ie, "cudaGraphInstantiate");
    }
    b->graph = gr;
    b->g_lam = d_lambda;
    b->g_vec = d_vectors;
    b->g_iters = d_iters;
  }
  BATCH_CUDA(cudaGraphLaunch(b->gexec, s));
  amm::count_launch(b->wide_count > 0 ? 2 : 1);
  return AMM_OK;
}

int amm_batch_run_each(amm_batch* b, double* d_lambda, float* d_vectors, int32_t* d_iters,
                       void* stream) {
  if (!b || !d_lambda || !d_vectors || !d_iters) return AMM_ERR_INVALID_ARGUMENT;
  Guard g(b->device);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  int rc = autotune(b, d_lambda, d_vectors, d_iters, s);
  if (rc) return rc;
  // one single-CTA launch per matrix; each reads its matrix index from a one-entry slice of
  // the order array
  for (int64_t i = 0; i < b->count; ++i) {
    rc = launch(b, b->variant, b->cluster, b->cluster, d_lambda, d_vectors, d_iters,
                (int)b->cfg.max_iter, b->d_order + i, 1, s);
    if (rc) return rc;
  }
  return AMM_OK;
}

int amm_batch_grad(amm_batch* b, const float* d_vectors, void* const* grad_ptrs,
                   const int64_t* grad_ld, const float* d_scale, void* stream) {
  if (!b || !d_vectors || !grad_ptrs || !grad_ld) return AMM_ERR_INVALID_ARGUMENT;
  for (int64_t i = 0; i < b->count; ++i) {
    if (!grad_ptrs[i] || grad_ld[i] < b->mats[i].m) return AMM_ERR_INVALID_ARGUMENT;
  }
  Guard g(b->device);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  BATCH_CUDA(cudaMemcpyAsync(b->d_grads, grad_ptrs, sizeof(void*) * b->count,
                             cudaMemcpyHostToDevice, s));
  BATCH_CUDA(cudaMemcpyAsync(b->d_grad_ld, grad_ld, sizeof(int64_t) * b->count,
                             cudaMemcpyHostToDevice, s));
  amm::batch::GradArgs a{};
  a.mats = b->d_mats;
  a.col_start = b->d_col_start;
  a.count = (int32_t)b->count;
  a.vec = d_vectors;
  a.grads = b->d_grads;
  a.grad_ld = b->d_grad_ld;
  a.scale = d_scale;
  // one warp per contiguous range of columns; a grid of the CTAs resident at once, 8 warps each
  int max_m = 1;
  for (const auto& M : b->mats) max_m = std::max(max_m, (int)M.m);
  a.vs_len = (max_m + 3) / 4 * 4;
  const size_t smem = sizeof(float) * 8 * (size_t)a.vs_len +
                      (b->count <= amm::batch::kGradSmemMats
                           ? sizeof(int64_t) * (size_t)(b->count + 1) : 0);
  if (smem > 48 * 1024)
    BATCH_CUDA(cudaFuncSetAttribute(amm::batch::grad_kernel,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  BATCH_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, amm::batch::grad_kernel, 256,
                                                           smem));
  const int64_t warps = b->total_cols;  // at least one column per warp
  int64_t blocks = (warps + 7) / 8;
  blocks = std::min<int64_t>(blocks, (int64_t)b->nsm * std::max(per_sm, 1));
  amm::batch::grad_kernel<<<(int)blocks, 256, smem, s>>>(a);
  amm::count_launch(1);
  BATCH_CUDA(cudaGetLastError());
  // (the pointer arrays come from pageable host memory: the copies above were staged before
  // they returned, so the caller's arrays may go at once)
  return AMM_OK;
}

int amm_batch_set_matrices(amm_batch* b, const amm_batch_matrix* mats, int64_t count,
                           void* stream) {
  if (!b || !mats || count != b->count) return AMM_ERR_INVALID_ARGUMENT;
  for (int64_t i = 0; i < count; ++i) {
    const amm_batch_matrix& x = mats[i];
    if (!x.A || x.m != b->mats[i].m || x.n != b->mats[i].n || x.ld < x.m)
      return AMM_ERR_INVALID_ARGUMENT;
    if ((reinterpret_cast<uintptr_t>(x.A) & 15) != 0 || (x.ld % 4) != 0) return AMM_ERR_ALIGNMENT;
  }
  // the new descriptors (and tensor maps) are formed first, so that a failure leaves the
  // context bound to the old matrices as a whole
  std::vector<Mat> ms = b->mats;
  for (int64_t i = 0; i < count; ++i) {
    ms[i].A = static_cast<const float*>(mats[i].A);
    ms[i].ld = mats[i].ld;
  }
  std::vector<CUtensorMap> tm;
  if (b->d_tmaps && !encode_tensor_maps(ms, tm)) return fail(cudaErrorInvalidValue, "tensor maps");
  b->mats.swap(ms);
  if (b->d_tmaps) b->h_tmaps.swap(tm);
  Guard g(b->device);
  // pageable sources: each copy is staged before the call returns, then stream-ordered
  BATCH_CUDA(cudaMemcpyAsync(b->d_mats, b->mats.data(), sizeof(Mat) * count,
                             cudaMemcpyHostToDevice, reinterpret_cast<cudaStream_t>(stream)));
  if (b->d_tmaps)
    BATCH_CUDA(cudaMemcpyAsync(b->d_tmaps, b->h_tmaps.data(), sizeof(CUtensorMap) * count,
                               cudaMemcpyHostToDevice, reinterpret_cast<cudaStream_t>(stream)));
  return AMM_OK;
}

int amm_batch_record(amm_batch* b, float* d_cdf, uint32_t* d_picks, int64_t products) {
  if (!b || products < 0 || products > (1 << 20) || (d_picks && products == 0))
    return AMM_ERR_INVALID_ARGUMENT;
  if ((d_cdf || d_picks) && !b->amm) return AMM_ERR_INVALID_ARGUMENT;
  b->rec_cdf = d_cdf;
  b->rec_picks = d_picks;
  b->rec_products = d_picks ? (int)products : 0;
  // the captured graph holds the launch arguments by value
  Guard g(b->device);
  if (b->gexec) cudaGraphExecDestroy(b->gexec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->gexec = nullptr;
  b->graph = nullptr;
  return AMM_OK;
}

int amm_batch_tile_choice(amm_batch* b, int32_t* k_out, int32_t* gc_out, int32_t* cl_out) {
  if (!b || !k_out || !gc_out) return AMM_ERR_INVALID_ARGUMENT;
  if (b->variant < 0) return AMM_ERR_NOT_READY;
  *k_out = amm::batch::kVariants[b->variant].K;
  *gc_out = amm::batch::kVariants[b->variant].GC;
  if (cl_out) *cl_out = b->cluster;
  return AMM_OK;
}

int amm_batch_wide_plan(amm_batch* b, int32_t* count, int32_t* cluster_size, int32_t* ctas,
                        float* ms) {
  if (!b || !count || !cluster_size || !ctas || !ms) return AMM_ERR_INVALID_ARGUMENT;
  if (b->variant < 0) return AMM_ERR_NOT_READY;
  *count = b->wide_count;
  *cluster_size = b->wide_count > 0 ? b->wide_cluster : 0;
  *ctas = b->wide_count > 0 ? b->wide_grid : 0;
  *ms = b->wide_ms;
  return AMM_OK;
}

}  // extern "C"
