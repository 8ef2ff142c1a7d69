// Reference-kernel harness: TEST INFRASTRUCTURE ONLY.
//
// Drives the reference's OWN drivers and kernels (Takuya-Okuyama/eigenvalueComputation_by_AMM,
// included read-only from the reference checkout with -I at build time; see oracle/Makefile)
// on caller-supplied inputs, so that the CUDA library and the numpy oracle can be compared
// with the reference itself on a B200.  Nothing here is part of the product; the built
// library lands in oracle/_ref/ and is loaded only by tests and fixture generators.
//
// The reference only works on square, column-major m x m matrices (m a multiple of 128,
// c a multiple of 8, c <= m); the entry points check those limits and return -1 otherwise.
// Each entry point builds the reference's host_memory / device_memory exactly as main()
// does (AMM.cu:74-95), replaces the generated matrix and the xorshift states with the
// caller's, recomputes the column norms and ||alpha||^2 the way write_data() does
// (device_memory.h:316-337), and then calls the reference code.

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>
#include <unistd.h>
#include <sys/stat.h>

#include "common.h"
#include "powerMethod_by_exact.cuh"
#include "powerMethod_by_previous.cuh"
#include "powerMethod_by_proposed.cuh"
#include "powerMethod_by_proposed_v2.cuh"

namespace {

struct Cwd {
  // The reference opens data/exact_eigenvector and result/... relative to the working
  // directory (device_memory.h:246-275); run it inside a private temporary directory.
  // Its constructor also indexes the last '/'-separated part of -filepath
  // (device_memory.h:256-259), which is out of range when no -filepath is given, so the
  // matrix is always handed over through the reference's own file loader: a uint32 size
  // header followed by size*size floats (host_memory.h:143-159, device_memory.h:369-401).
  std::string old_dir, dir;
  Cwd(const double *vstar, int64_t m, const float *A) {
    char buf[4096];
    if (getcwd(buf, sizeof(buf))) old_dir = buf;
    char tmpl[] = "/tmp/amm_ref_XXXXXX";
    char *d = mkdtemp(tmpl);
    dir = d ? d : "/tmp";
    if (chdir(dir.c_str()) != 0) return;
    mkdir("data", 0755);
    mkdir("result", 0755);
    std::vector<double> v(m, 0.0);
    if (vstar)
      for (int64_t i = 0; i < m; ++i) v[i] = vstar[i];
    FILE *f = fopen("data/exact_eigenvector", "wb");
    if (f) {
      fwrite(v.data(), sizeof(double), m, f);
      fclose(f);
    }
    // loader order: h_matrix[y*size + x] = file[y*size + x], i.e. the file holds dA itself
    f = fopen("matrix.bin", "wb");
    if (f) {
      const uint32_t sz = (uint32_t)m;
      fwrite(&sz, sizeof(uint32_t), 1, f);
      fwrite(A, sizeof(float), (size_t)m * (size_t)m, f);
      fclose(f);
    }
  }
  ~Cwd() {
    if (!old_dir.empty() && chdir(old_dir.c_str()) != 0) {
    }
    std::string cmd = "rm -rf '" + dir + "'";
    if (dir.rfind("/tmp/amm_ref_", 0) == 0 && system(cmd.c_str()) != 0) {
    }
  }
};

bool sizes_ok(int64_t m, int64_t c) {
  return m >= 128 && m % 128 == 0 && c >= 8 && c % 8 == 0 && c <= m;
}

std::vector<std::string> make_args(const char *kernel, int64_t m, int64_t c, int64_t step,
                                   int64_t vr_period, double vr_thr, int sanity, uint32_t seed) {
  std::vector<std::string> a = {"AMM", "-m", std::to_string(m), "-c", std::to_string(c),
                                "-step", std::to_string(step), "-kernel", kernel,
                                "-seed", std::to_string(seed), "-r", "1",
                                "-filepath", "matrix.bin"};
  if (vr_period > 0) {
    a.push_back("-vr");
    a.push_back(std::to_string(vr_period));
  }
  if (vr_thr > 0.0) {
    char b[64];
    snprintf(b, sizeof(b), "%.17g", vr_thr);
    a.push_back("-vr_adaptive");
    a.push_back(b);
  }
  if (sanity) a.push_back("-sanity");
  return a;
}

// write_data() has loaded A from matrix.bin and derived the norms and ||alpha||^2 from it;
// check the upload and replace the xorshift states with the caller's.
int load_inputs(host_memory &p, device_memory &dm, const float *A, const uint32_t *states) {
  std::vector<float> back((size_t)dm.m * dm.m);
  cudaMemcpy(back.data(), dm.dA, sizeof(float) * back.size(), cudaMemcpyDeviceToHost);
  if (memcmp(back.data(), A, sizeof(float) * back.size()) != 0) return -4;
  p.diagonal_offset = 0.0f;
  cudaMemcpy(dm.d_rnd, states, sizeof(uint32_t) * dm.m, cudaMemcpyHostToDevice);
  return cudaDeviceSynchronize() == cudaSuccess ? 0 : -3;
}

}  // namespace

extern "C" {

// Raw start vector the reference would draw for a given x0 seed: curandGenerateNormal of m
// values from a fresh default generator seeded with x0_seed (powerMethod_by_exact.cuh:32).
int ref_draw_x0(int64_t m, uint64_t x0_seed, float *x0_out) {
  curandGenerator_t g;
  float *d = nullptr;
  if (curandCreateGenerator(&g, CURAND_RNG_PSEUDO_DEFAULT) != CURAND_STATUS_SUCCESS) return -2;
  curandSetPseudoRandomGeneratorSeed(g, x0_seed);
  cudaMalloc(&d, sizeof(float) * m);
  curandGenerateNormal(g, d, m, 0.0, 1.0);
  cudaMemcpy(x0_out, d, sizeof(float) * m, cudaMemcpyDeviceToHost);
  cudaFree(d);
  curandDestroyGenerator(g);
  return cudaGetLastError() == cudaSuccess ? 0 : -3;
}

// The xorshift states the reference derives from -seed (device_memory.h:339-343).
int ref_seed_states(int64_t m, uint64_t seed, uint32_t *states_out) {
  curandGenerator_t g;
  uint32_t *d = nullptr;
  if (curandCreateGenerator(&g, CURAND_RNG_PSEUDO_DEFAULT) != CURAND_STATUS_SUCCESS) return -2;
  curandSetPseudoRandomGeneratorSeed(g, seed + 1234);
  cudaMalloc(&d, sizeof(uint32_t) * m);
  curandGenerate(g, d, m);
  cudaMemcpy(states_out, d, sizeof(uint32_t) * m, cudaMemcpyDeviceToHost);
  cudaFree(d);
  curandDestroyGenerator(g);
  return cudaGetLastError() == cudaSuccess ? 0 : -3;
}

// One call of powerMethod_by_<kernel>(p, dm, is_output=true) on the caller's A (m x m,
// column-major) and xorshift states (m values).  The start vector is drawn by the reference
// from a generator seeded with x0_seed (use ref_draw_x0 to get it).  Outputs: λ and err per
// step (the reference's d_eigs / d_errs), the final x and y, the per-column statistics, the
// FP32 CDF and inverse-probability weights of the last weighting used, the last sorted index
// set, the advanced states and the elapsed time of the whole call in ms (CUDA events, the
// reference's own per-step host syncs included).
int ref_power_method(const char *kernel, int64_t m, int64_t c, int64_t step, int64_t vr_period,
                     double vr_thr, int sanity, const float *A, uint64_t x0_seed,
                     const uint32_t *states, const double *vstar, double *eigs_out,
                     double *errs_out, float *x_out, float *y_out, float *alpha_out,
                     float *norm_out, float *normp_out, float *cdf_out, float *weight_out,
                     uint32_t *sorted_out, uint32_t *states_out, float *time_ms_out) {
  if (!sizes_ok(m, c) || step < 1) return -1;
  std::string k(kernel);
  if (k == "proposedAMM_v2" && (vr_period < 1 || step < vr_period)) return -1;
  Cwd cwd(vstar, m, A);
  auto args = make_args(kernel, m, c, step, vr_period, vr_thr, sanity, 7u);
  std::vector<char *> argv;
  for (auto &s : args) argv.push_back(const_cast<char *>(s.c_str()));
  host_memory p;
  if (!p.parser((int)argv.size(), argv.data())) return -1;
  int rc = 0;
  {
    device_memory dm(p);
    dm.write_data(p);
    rc = load_inputs(p, dm, A, states);
    if (rc) return rc;
    curandSetPseudoRandomGeneratorSeed(dm.gen, x0_seed);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    if (k == "exact")
      powerMethod_by_exact(p, dm, true);
    else if (k == "previousAMM")
      powerMethod_by_previous(p, dm, true);
    else if (k == "proposedAMM")
      powerMethod_by_proposed(p, dm, true);
    else if (k == "proposedAMM_v2")
      powerMethod_by_proposed_v2(p, dm, true);
    else
      rc = -1;
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (time_ms_out) *time_ms_out = ms;
    cudaDeviceSynchronize();
    if (eigs_out) cudaMemcpy(eigs_out, dm.d_eigs, sizeof(double) * step, cudaMemcpyDeviceToHost);
    if (errs_out) cudaMemcpy(errs_out, dm.d_errs, sizeof(double) * step, cudaMemcpyDeviceToHost);
    if (x_out) cudaMemcpy(x_out, dm.dx, sizeof(float) * m, cudaMemcpyDeviceToHost);
    if (y_out) cudaMemcpy(y_out, dm.dy, sizeof(float) * m, cudaMemcpyDeviceToHost);
    if (alpha_out) cudaMemcpy(alpha_out, dm.d_alpha, sizeof(float) * m, cudaMemcpyDeviceToHost);
    if (norm_out) cudaMemcpy(norm_out, dm.d_normA, sizeof(float) * m, cudaMemcpyDeviceToHost);
    if (normp_out)
      cudaMemcpy(normp_out, dm.d_normAprime, sizeof(float) * m, cudaMemcpyDeviceToHost);
    if (cdf_out) cudaMemcpy(cdf_out, dm.d_acc_weight, sizeof(float) * m, cudaMemcpyDeviceToHost);
    if (weight_out)
      cudaMemcpy(weight_out, dm.d_weight, sizeof(float) * m, cudaMemcpyDeviceToHost);
    if (sorted_out)
      cudaMemcpy(sorted_out, dm.d_sorted_pos, sizeof(uint32_t) * c, cudaMemcpyDeviceToHost);
    if (states_out) cudaMemcpy(states_out, dm.d_rnd, sizeof(uint32_t) * m, cudaMemcpyDeviceToHost);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (cudaDeviceSynchronize() != cudaSuccess) rc = -3;
  }
  return rc;
}

// Step-by-step AMM without variance reduction, dumping every step: the reference's
// square_of_A_by_previous / square_of_A_by_proposed (powerMethod_by_previous.cuh:7-98,
// powerMethod_by_proposed.cuh:7-103) followed by dotProduct_and_generate_x (common.h:89-154),
// started from normalize(x0) (common.h:156-183).  For "proposedAMM" z = A·alpha and
// v = z - ||alpha||^2 are prepared as powerMethod_by_proposed does (:343-364).
// sorted_out: nsteps*c, tmp_out: nsteps*c, y_out: nsteps*m, eigs_out: nsteps, cdf_out and
// weight_out: m (after the first step), states_out: m.
int ref_amm_steps(const char *kernel, int64_t m, int64_t c, int64_t nsteps, int sanity,
                  const float *A, const float *x0, const uint32_t *states, uint32_t *sorted_out,
                  float *tmp_out, float *y_out, double *eigs_out, float *cdf_out,
                  float *weight_out, uint32_t *states_out) {
  if (!sizes_ok(m, c) || nsteps < 1) return -1;
  std::string k(kernel);
  if (k != "previousAMM" && k != "proposedAMM") return -1;
  Cwd cwd(nullptr, m, A);
  auto args = make_args(kernel, m, c, nsteps, 0, 0.0, sanity, 7u);
  std::vector<char *> argv;
  for (auto &s : args) argv.push_back(const_cast<char *>(s.c_str()));
  host_memory p;
  if (!p.parser((int)argv.size(), argv.data())) return -1;
  int rc = 0;
  {
    device_memory dm(p);
    dm.write_data(p);
    rc = load_inputs(p, dm, A, states);
    if (rc) return rc;
    cublasSetStream(dm.handle, dm.stream_1);
    if (k == "proposedAMM") {
      cublasSgemv(dm.handle, CUBLAS_OP_N, p.m, p.m, &p.const_one, dm.dA, p.m, dm.d_alpha, 1,
                  &p.const_zero, dm.dz, 1);
      generate_v<512><<<1, 512, 0, dm.stream_1>>>(dm.dv, dm.dz, p.alpha2, dm.m);
    }
    cudaMemcpy(dm.dx, x0, sizeof(float) * m, cudaMemcpyHostToDevice);
    normalize<512><<<1, 512, 0, dm.stream_1>>>(dm.dx, dm.m);
    for (int64_t i = 0; i < nsteps; ++i) {
      if (k == "previousAMM")
        square_of_A_by_previous(dm, p.sanity_check);
      else
        square_of_A_by_proposed(dm, p.sanity_check);
      cudaStreamSynchronize(dm.stream_1);
      if (sorted_out)
        cudaMemcpy(sorted_out + i * c, dm.d_sorted_pos, sizeof(uint32_t) * c,
                   cudaMemcpyDeviceToHost);
      if (tmp_out) cudaMemcpy(tmp_out + i * c, dm.dtmp, sizeof(float) * c, cudaMemcpyDeviceToHost);
      if (y_out) cudaMemcpy(y_out + i * m, dm.dy, sizeof(float) * m, cudaMemcpyDeviceToHost);
      dotProduct_and_generate_x<64><<<1, 64, 0, dm.stream_1>>>(
          dm.d_dots, dm.d_eigs + i, dm.d_errs + i, dm.dx, dm.d_eigenvector, dm.m);
      cudaStreamSynchronize(dm.stream_1);
    }
    if (eigs_out) cudaMemcpy(eigs_out, dm.d_eigs, sizeof(double) * nsteps, cudaMemcpyDeviceToHost);
    if (cdf_out) cudaMemcpy(cdf_out, dm.d_acc_weight, sizeof(float) * m, cudaMemcpyDeviceToHost);
    if (weight_out)
      cudaMemcpy(weight_out, dm.d_weight, sizeof(float) * m, cudaMemcpyDeviceToHost);
    if (states_out) cudaMemcpy(states_out, dm.d_rnd, sizeof(uint32_t) * m, cudaMemcpyDeviceToHost);
    if (cudaDeviceSynchronize() != cudaSuccess) rc = -3;
  }
  return rc;
}

// pick_index alone (device_memory.h:516-545) on a caller-supplied FP32 CDF of length n and
// c states: the bit-exactness anchor for the sampler.  idx_out: c, states_out: c.
int ref_pick_index(int64_t n, int64_t c, const float *cdf, const uint32_t *states,
                   uint32_t *idx_out, uint32_t *states_out) {
  if (n < 1 || c < 1) return -1;
  float *d_cdf = nullptr;
  uint32_t *d_st = nullptr, *d_idx = nullptr;
  cudaMalloc(&d_cdf, sizeof(float) * n);
  cudaMalloc(&d_st, sizeof(uint32_t) * c);
  cudaMalloc(&d_idx, sizeof(uint32_t) * c);
  cudaMemcpy(d_cdf, cdf, sizeof(float) * n, cudaMemcpyHostToDevice);
  cudaMemcpy(d_st, states, sizeof(uint32_t) * c, cudaMemcpyHostToDevice);
  pick_index<<<DIV_CEIL((uint64_t)c, (uint64_t)128), 128>>>(d_idx, d_st, d_cdf, (uint64_t)n,
                                                            (uint64_t)c);
  cudaMemcpy(idx_out, d_idx, sizeof(uint32_t) * c, cudaMemcpyDeviceToHost);
  cudaMemcpy(states_out, d_st, sizeof(uint32_t) * c, cudaMemcpyDeviceToHost);
  int rc = cudaDeviceSynchronize() == cudaSuccess ? 0 : -3;
  cudaFree(d_cdf);
  cudaFree(d_st);
  cudaFree(d_idx);
  return rc;
}

// The reference's matrix generator (device_memory.h:360-433) for -matrixType `type` and seed
// `seed` on an m x m matrix: A_out receives dA (column-major) with its diagonal offset added,
// *offset_out the offset.
int ref_generate(const char *type, int64_t m, uint32_t seed, float *A_out, float *offset_out) {
  if (!sizes_ok(m, 8)) return -1;
  std::vector<float> zero((size_t)m * (size_t)m, 0.0f);
  Cwd cwd(nullptr, m, zero.data());
  auto args = make_args("exact", m, 8, 1, 0, 0.0, 0, seed);
  std::vector<char *> argv;
  for (auto &s : args) argv.push_back(const_cast<char *>(s.c_str()));
  host_memory p;
  if (!p.parser((int)argv.size(), argv.data())) return -1;
  int rc = 0;
  {
    // constructed with -filepath (its result-file naming needs one), then write_data() runs
    // with the path cleared, which takes the reference's -matrixType generator branch
    device_memory dm(p);
    p.filepath = "";
    p.matrixType = std::string(type);
    dm.write_data(p);
    cudaDeviceSynchronize();
    if (offset_out) *offset_out = p.diagonal_offset;
    if (A_out) cudaMemcpy(A_out, dm.dA, sizeof(float) * m * m, cudaMemcpyDeviceToHost);
    if (cudaDeviceSynchronize() != cudaSuccess) rc = -3;
  }
  return rc;
}

}  // extern "C"
