// Internal declarations shared by the kernels (amm_kernels.cu) and the host side (amm_api.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace amm {

// Step kinds, identical to enum amm_step_kind in include/amm.h.
enum StepKind : int32_t { kExactMemo = 0, kExact = 1, kPrevious = 2, kProposed = 3 };
enum Method : int32_t { kMethodExact = 0, kMethodPrevious = 1, kMethodProposed = 2, kMethodProposedV2 = 3 };

// Device status bits (ORed into Buffers::status).
enum DevStatus : uint32_t { kDevTimeout = 1u, kDevNonFinite = 2u, kDevBadIndex = 4u };

constexpr int kMaxThreads = 512;   // panel kernel block size limit
constexpr int kGcMax = 8;          // columns per pipeline stage, upper bound
constexpr int kSeg = 32;           // fine-search window of the sampler (elements)
constexpr int kCoarseMax = 2048;   // coarse CDF table entries held in shared memory
constexpr int kCdfTile = 1024;     // columns per block of the CDF construction
// AMM work lists drawn ahead.  The picks of an AMM step depend only on the sampling states and
// the CDF, never on x, so the lists of up to kListWindow consecutive AMM steps are drawn and
// compacted together before the first of them (one refill every kListWindow steps); list a of a
// call (its a-th AMM step) lives in slot a % kListWindow.  16 covers the solves the bench's
// schedules need (7 to 9 steps) in one persistent step launch; a slot costs 4·n + 16·c bytes.
constexpr int kListWindow = 16;

// Iteration state, by iteration parity: a launch of the step kernel covering steps [i0, i1)
// reads st[i0 & 1] and leaves the state after its last step in st[i1 & 1] (the sampler's refill
// ahead of step i reads st[i & 1]); inside the launch every CTA keeps its own copy.
struct IterState {
  int32_t mode;        // StepKind of this iteration
  int32_t last_exact;  // proposed AMM: index of the last VR step
  int32_t done;        // early stop reached: later kernels of the call do nothing
  int32_t used;        // work lists consumed by the call's AMM steps so far
  int32_t drawn;       // work lists drawn so far: lists [used, drawn) are pending
  int32_t steps_run;   // completed steps
  int32_t distinct;    // distinct columns of the last AMM product (written by the panel kernel)
  int32_t memo_zero;   // the memo pair is zero (call start, until the first VR step)
  float scale;         // x_i = scale * y_{i-1} (FP32 multiply)
  float pad2;
  double cos_prev;     // cos of the previous step (adaptive VR)
  double lam_prev;     // λ of the previous step (tolerance stop)
};
static_assert(sizeof(IterState) == 56, "the trace read copies 56 bytes of state");

// Static description of one power-method call, passed by value to the kernels.
struct CallCfg {
  int32_t method;
  int32_t vr_period;
  double vr_thr;
  double tol;
  int32_t variance_reduction;
  int32_t sanity;      // sanity mode active (sanity && c == n)
  int32_t uses_amm;    // the call draws samples at all
  int32_t step;
  int32_t ext_list;    // the (single) AMM step's work list in slot 0 comes from the caller or
                       // from a sharded draw: the context draws nothing and keeps its states
};

// Every device buffer of a context.
struct Buffers {
  // matrix
  const void* A;
  int64_t ld;
  int32_t m, n, c;
  int32_t dtype;       // 0 FP32, 1 BF16
  int32_t cdf_f32;     // 1: FP32 CDF and target
  int32_t nsm;         // partial sums written by the panel kernel (one per cluster)
  // per-column statistics (n)
  float* alpha;
  float* norm;
  float* normp;
  // sampling tables per weighting (0 = norm, 1 = normp)
  double* cdf64[2];
  float* cdf32[2];
  float* wts[2];
  double* coarse64[2];
  float* coarse32[2];
  int32_t seg;         // elements per coarse segment (power of two >= kSeg)
  int32_t ncoarse;     // full segments = n / seg
  int32_t chunk_shift; // log2 of the distinct-count chunk
  int32_t nchunks;
  // vectors (m)
  float* z;
  float* v;
  float* y[2];         // y[i & 1] = y_i; y[1] holds the raw start vector for i = 0
  float* x_memo;
  float* y_memo;
  double* vstar;       // may be null
  int32_t has_vstar;
  // sampling
  uint32_t* states[2];   // xorshift states (c used); states[0]: committed at the call start
  uint32_t* count[kListWindow];    // per slot: per-column multiplicity of the picks (n)
  uint32_t* chunk[kListWindow];    // per slot: distinct columns per chunk (nchunks)
  uint32_t* samples[kListWindow];  // per slot: raw picks in draw order (c)
  uint32_t* distinct_idx;   // sorted distinct indices of the last AMM product (c)
  uint32_t* distinct_mult;  // their multiplicities (c)
  // work list of each slot: sorted distinct columns with their coefficient data, built by
  // compact_kernel
  uint32_t* wl_col[kListWindow];  // c
  float* wl_wm[kListWindow];      // c: w_j · multiplicity
  float* wl_al[kListWindow];      // c: α_j
  uint32_t* wl_count;             // kListWindow: number of distinct columns of each slot
  // partial sums
  float* partials;     // nsm x m
  float* spart;        // nsm  (Σ α_k t_k of each CTA, proposed)
  double* spart64;     // nsm  (Σ α_j² of each CTA, set-up)
  double2* colsum;     // n (Σa, Σa²) of each column from the set-up pass
  double* rpart;       // nsm x 4 (x·y, y·y, y·v*, z·dx) of each CTA
  uint32_t* ticket;    // [2]: grid-barrier arrivals of the step kernel and the set-up pass;
                       // [3]: the wait probe's barrier; [0], [1]: spare
  double* alpha2;      // ‖α‖²
  float* colvec;       // n floats of scratch (vᵀA for the gradient)
  double* cdf_tsum;    // 2 x ceil(n/kCdfTile) tile sums of the CDF build
  // iteration state and traces
  IterState* st;       // [2]
  double* eigs;
  double* errs;
  double* coss;
  int32_t* kinds;
  int32_t* distinct_hist;
  unsigned long long* tstamp;  // step+1 entries: [0] start, [i+1] end of step i
  uint32_t* status;
};

// Launch geometry of the panel kernel for a given (m, dtype).
struct PanelGeom {
  int dtype;        // 0 FP32, 1 BF16
  int cluster;      // CTAs per thread-block cluster (1: no clusters).  The CTAs of a cluster
                    // pre-sum their partial y through distributed shared memory: rank r sums
                    // rows [r*m/cluster, (r+1)*m/cluster) of the cluster's partials
  int rows;         // rows each CTA streams (all m)
  int nclusters;    // clusters launched (= partial y vectors written per step)
  int grid;         // CTAs launched = nclusters * cluster (one per SM, all resident)
  int threads;      // consumer threads (a producer warp is added)
  int slots;        // 16-byte vector slots per consumer thread (R)
  int elems;        // elements per 16-byte vector (E)
  int colbytes;     // bytes of one column slice = rows * elem_size
  int gc;           // columns per stage (group)
  int nstages;
  int stage_bytes;  // gc * colbytes
  int stage_area;   // bytes reserved for the stages
  int smem_bytes;   // dynamic shared memory (set-up variant, the larger one)
  int wl_cap;       // work-list capacity per cluster
};

// cluster: requested CTAs per cluster (1, 2, 4 or 8; falls back to 1 where the shape or the
// residency does not allow it).
bool panel_geometry(int m, int dtype, int c, int n, int nsm, int cluster, PanelGeom* g);
// CTAs per cluster the step kernel is asked to use (AMM_PANEL_CLUSTER, default 1).
int panel_cluster_request();
// One CTA of the step kernel and of the set-up pass fits on an SM with the geometry's
// shared-memory carve (the persistent grids need every CTA resident at once); with clusters,
// fixes the grid to the clusters that fit at once (false if fewer than half the SMs).
bool panel_coresident(PanelGeom* g, int nsm);

// ---- launchers (amm_kernels.cu); each returns the cudaError_t of the launch ----
// Set-up pass over A (amm_panel.cu): column statistics (α, ‖A_j‖, ‖A_j − α_j‖), z = A·α,
// v = z − ‖α‖² and ‖α‖², in one read of A.
cudaError_t launch_setup_panel(const Buffers& b, const PanelGeom& g, cudaStream_t s);
// Build the CDFs, weights and coarse tables of both weightings (or one if which >= 0,
// keeping an imported CDF when keep_cdf is set).
cudaError_t launch_build_cdf(const Buffers& b, int which, int keep_cdf, int sanity, cudaStream_t s);
// Start of a call: x0 into y[1], scale, initial state, first picks.
// no_normalize: use x0 as x_0 unscaled (single-product entry points).
cudaError_t launch_init(const Buffers& b, const CallCfg& cc, const float* x0, int no_normalize,
                        cudaStream_t s);
// Refill of the work-list window ahead of step iter (iter % kListWindow == 0): draw the picks of
// the lists not yet drawn among the next kListWindow AMM steps.
cudaError_t launch_sample(const Buffers& b, const CallCfg& cc, int iter, cudaStream_t s);
// Record a CUDA failure for amm_last_cuda_error and return AMM_ERR_CUDA.
int record_cuda_failure(cudaError_t e, const char* what);
// Build the sorted distinct work lists of the picks just drawn (same decision as sample_kernel).
cudaError_t launch_compact(const Buffers& b, const CallCfg& cc, int iter, cudaStream_t s);
// Steps [iter, iter_end) of a call in one persistent launch (amm_panel.cu): per step the
// product, the grid-wide reduction of the partials into y, the Rayleigh quotient and the next
// step's state.
cudaError_t launch_iter_panel(const Buffers& b, const PanelGeom& g, const CallCfg& cc, int iter,
                              int iter_end, cudaStream_t s);
// x_final = scale * y_last into dst (length m); y_last into ydst (optional); commits the
// sampling states to states[0] and clears any pending picks.
cudaError_t launch_finalize(const Buffers& b, const CallCfg& cc, float* xdst, float* ydst,
                            cudaStream_t s);
// Standalone helpers.
cudaError_t launch_normalize(float* x, int m, cudaStream_t s);
// Device-to-device copy of n floats by a kernel (a memcpy when unaligned).
cudaError_t launch_copy(float* dst, const float* src, int n, cudaStream_t s);
cudaError_t launch_clock(unsigned long long* out, cudaStream_t s);
// The failure path of the bounded waits, on purpose (one CTA; out: 3 words, see the kernel).
cudaError_t launch_wait_probe(uint32_t* status, uint32_t* counter, uint32_t* out,
                              cudaStream_t s);
cudaError_t launch_rayleigh(const float* x_in, float* x_out, const float* y, const double* vstar,
                            int m, double* out3, cudaStream_t s);
cudaError_t launch_sample_only(const Buffers& b, int which, uint32_t* idx, cudaStream_t s);
cudaError_t launch_expand_sorted(const Buffers& b, const int32_t* d_cd, uint32_t* out,
                                 cudaStream_t s);
cudaError_t launch_grad(const Buffers& b, const float* v, float* grad, int64_t ldg,
                        cudaStream_t s);
// Caller-supplied work list in slot 0 (count entries of wl_col[0], wl_wm[0]): α of each listed
// column into wl_al[0]; an index outside [0, n) becomes column 0 with weight 0 and sets
// kDevBadIndex.
cudaError_t launch_gather_alpha(const Buffers& b, int64_t count, cudaStream_t s);
// One rank's work list (slot 0) from a draw over a column-sharded matrix's global CDF: picks in
// [col0, col0 + n) of the c picks drawn from st_in (advanced into st_out, may alias).
cudaError_t launch_shard_worklist(const Buffers& b, const double* cdf, int n_global, int col0,
                                  const uint32_t* st_in, uint32_t* st_out, int c, cudaStream_t s);

// Count of this library's launches (for the bench's gpu_launches field).
void count_launch(int k = 1);
int64_t launch_count();
// Programmatic dependent launch in use (AMM_PDL=0 turns it off).
bool pdl_enabled();

}  // namespace amm
