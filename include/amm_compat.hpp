// amm_compat.hpp — the reference's C++ host interface over the C ABI of libamm.
//
// Reference-style host code (Takuya-Okuyama/eigenvalueComputation_by_AMM) includes this header
// instead of common.h / powerMethod_by_*.cuh and links -lamm.  It keeps the names, argument
// meanings and call order of the reference:
//   host_memory                 parameters and the flag parser      (host_memory.h:23-192)
//   device_memory               buffers, generators, result file     (device_memory.h:116-498)
//   powerMethod_by_exact / _previous / _proposed / _proposed_v2(p, dm, is_output)
//                                                                    (powerMethod_by_*.cuh)
//   square_of_A_by_previous / _proposed(dm, sanity)                 (powerMethod_by_previous.cuh:7,
//                                                                     powerMethod_by_proposed.cuh:7)
// Differences, all deliberate: every libamm call returns a status and a failure throws
// amm_compat::error (the reference checks nothing); the matrix may be rectangular (m x n);
// dm.dA is a device buffer the caller may fill directly; the whole iteration loop runs on the
// device without a host round trip per step, so the per-step times in the result file come
// from device timestamps rather than a host event sync per step.
#ifndef AMM_COMPAT_HPP_
#define AMM_COMPAT_HPP_

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "amm.h"

namespace amm_compat {

struct error : std::runtime_error {
  int status;
  error(int s, const std::string& where)
      : std::runtime_error(where + ": " + amm_status_string(s) +
                           (s == AMM_ERR_CUDA ? std::string(" (") + amm_last_cuda_error() + ")"
                                              : std::string())),
        status(s) {}
};

inline void check(int s, const char* where) {
  if (s != AMM_OK) throw error(s, where);
}

}  // namespace amm_compat

// ---------------------------------------------------------------------------------------------
// host_memory: the reference's parameters (host_memory.h:26-50) and flags (:65-130)
// ---------------------------------------------------------------------------------------------
class host_memory {
 public:
  uint64_t original_m = 128;
  uint64_t m = 128;
  uint64_t n = 0;  // columns; 0 = square (the reference's only case)
  uint32_t c = 0;
  uint64_t step = 10;
  uint64_t vr_period = 0;
  std::string str_vr_adaptive_threshold;
  double vr_adaptive_threshold = 0.0;
  std::string kernel = "exact";
  std::string matrixType = "gaussian_0.0_1.0";
  std::string filepath;
  int verbose = 0;
  uint32_t nreps = 10;
  uint32_t seed = (uint32_t)time(nullptr);
  float alpha2 = 0.0f;
  float diagonal_offset = 0.0f;
  bool sanity_check = false;
  bool variance_reduction = false;
  bool display = false;
  bool bf16 = false;  // extension: store A in BF16 (-bf16)

  // Same flags as host_memory::parser (host_memory.h:65-187); m is rounded up to a multiple
  // of 128 and c defaults to m as there.  Returns false on an invalid -kernel or an unreadable
  // -filepath.
  bool parser(int argc, char** argv) {
    for (int i = 1; i < argc; ++i) {
      const std::string a = argv[i];
      auto next = [&]() -> const char* { return i + 1 < argc ? argv[++i] : ""; };
      if (a == "-m") {
        m = (uint64_t)std::atoll(next());
        m = (m + 127) / 128 * 128;
        original_m = m;
      } else if (a == "-n") {
        n = (uint64_t)std::atoll(next());
      } else if (a == "-c") {
        c = (uint32_t)std::atoi(next());
      } else if (a == "-r") {
        nreps = (uint32_t)std::atoi(next());
      } else if (a == "-step") {
        step = (uint64_t)std::atoll(next());
      } else if (a == "-kernel") {
        kernel = next();
      } else if (a == "-matrixType") {
        matrixType = next();
      } else if (a == "-filepath") {
        filepath = next();
      } else if (a == "-seed") {
        seed = (uint32_t)std::atoi(next());
      } else if (a == "-sanity") {
        sanity_check = true;
      } else if (a == "-display") {
        display = true;
      } else if (a == "-vr") {
        vr_period = (uint64_t)std::atoll(next());
        variance_reduction = vr_period > 0;
      } else if (a == "-vr_adaptive") {
        str_vr_adaptive_threshold = next();
        vr_adaptive_threshold = std::atof(str_vr_adaptive_threshold.c_str());
        variance_reduction = vr_adaptive_threshold > 0.0;
      } else if (a == "-verbose") {
        verbose = std::atoi(next());
      } else if (a == "-bf16") {
        bf16 = true;
      } else {
        printf("[warning] unknown parameter: %s\n", argv[i]);
      }
    }
    if (kernel == "exact") {
      sanity_check = false;
    } else if (kernel != "previousAMM" && kernel != "proposedAMM" && kernel != "proposedAMM_v2") {
      printf("[error] '-kernel %s' is not valid.\n", kernel.c_str());
      return false;
    }
    if (!filepath.empty()) {
      std::ifstream ifs(filepath, std::ios::in | std::ios::binary);
      if (ifs.fail()) {
        fprintf(stderr, "Failed to open file.\n");
        return false;
      }
      uint32_t val = 0;
      ifs.read(reinterpret_cast<char*>(&val), sizeof(uint32_t));
      original_m = val;
      m = (val + 127ull) / 128 * 128;
    }
    if (n == 0) n = m;
    if (kernel == "exact") c = (uint32_t)n;
    if (c == 0) c = (uint32_t)n;
    return true;
  }
};

// ---------------------------------------------------------------------------------------------
// device_memory: owns the libamm context, the device matrix and the result file
// ---------------------------------------------------------------------------------------------
struct device_memory {
  amm_ctx* ctx = nullptr;
  void* dA = nullptr;  // m x n column-major, FP32 or BF16 (ld = m)
  float* dx = nullptr;  // start vector buffer (length m)
  uint64_t m = 0, n = 0, original_m = 0, c = 0;
  std::string kernel;
  bool is_init = true;
  cudaStream_t stream_1 = nullptr;
  std::ofstream ofs_output;
  uint32_t seed = 0;
  // Values drawn so far from the reference's single cuRAND generator, which re-seeding does
  // not rewind: the matrix (size²) when generated, then the m states; the start vectors follow.
  uint64_t gen_pos = 0;

  explicit device_memory(host_memory& p) {
    m = p.m;
    n = p.n ? p.n : p.m;
    original_m = p.original_m;
    c = p.c;
    seed = p.seed;
    kernel = p.kernel;
    amm_config cfg;
    amm_config_default(&cfg);
    cfg.m = (int64_t)m;
    cfg.n = (int64_t)n;
    cfg.c = (int64_t)c;
    cfg.step = (int64_t)p.step;
    cfg.vr_period = (int64_t)p.vr_period;
    cfg.vr_adaptive_threshold = p.variance_reduction ? p.vr_adaptive_threshold : 0.0;
    if (!p.variance_reduction) cfg.vr_period = 0;
    cfg.dtype = p.bf16 ? AMM_BF16 : AMM_F32;
    cfg.cdf_precision = AMM_CDF_F32;  // the reference's FP32 CDF and target
    cfg.sanity = p.sanity_check ? 1 : 0;
    int dev = 0;
    cudaGetDevice(&dev);
    amm_compat::check(amm_create(&ctx, &cfg, dev), "amm_create");
    const size_t es = p.bf16 ? 2 : 4;
    if (cudaMalloc(&dA, es * m * n) != cudaSuccess || cudaMalloc((void**)&dx, sizeof(float) * m))
      throw amm_compat::error(AMM_ERR_OUT_OF_MEMORY, "device_memory");
    cudaStreamCreate(&stream_1);
    // the exact eigenvector for the error column, as the reference reads it (:246-254)
    std::vector<double> v(m, 0.0);
    std::ifstream ifs("data/exact_eigenvector", std::ios::in | std::ios::binary);
    if (ifs.good()) {
      ifs.read(reinterpret_cast<char*>(v.data()), sizeof(double) * original_m);
      double* dv = nullptr;
      cudaMalloc((void**)&dv, sizeof(double) * m);
      cudaMemcpy(dv, v.data(), sizeof(double) * m, cudaMemcpyHostToDevice);
      amm_compat::check(amm_set_eigenvector(ctx, dv, nullptr), "amm_set_eigenvector");
      cudaDeviceSynchronize();
      cudaFree(dv);
    }
    // result file name (:256-275)
    std::string base = p.filepath;
    const size_t slash = base.find_last_of('/');
    if (slash != std::string::npos) base = base.substr(slash + 1);
    std::string path = "result/eigenvalues_by_" + kernel + "_" + base + "_r=" +
                       std::to_string(p.nreps) + "_step=" + std::to_string(p.step);
    if (p.kernel != "exact") {
      path += "_c=" + std::to_string(p.c);
      path += p.vr_adaptive_threshold == 0.0 ? "_vr=" + std::to_string(p.vr_period)
                                             : "_vr=adaptive-" + p.str_vr_adaptive_threshold;
    }
    path += ".binary";
    ofs_output.open(path, std::ios::out | std::ios::binary);
  }

  ~device_memory() {
    ofs_output.close();
    if (ctx) amm_destroy(ctx);
    cudaFree(dA);
    cudaFree(dx);
    if (stream_1) cudaStreamDestroy(stream_1);
  }

  device_memory(const device_memory&) = delete;
  device_memory& operator=(const device_memory&) = delete;

  // Set by a caller that filled dA itself; otherwise write_data loads or generates A.
  bool matrix_ready = false;

  // The matrix part of write_data (:316-337 with generate_matrix, :360-433): the -filepath
  // covariance file (padded with zeros to m), or the -matrixType generator seeded with -seed
  // (p.diagonal_offset receives its offset).  FP32 storage only; with -bf16 the caller fills
  // dA and sets matrix_ready.
  void load_or_generate(host_memory& p) {
    if (p.bf16) throw amm_compat::error(AMM_ERR_UNSUPPORTED, "write_data: fill dA for -bf16");
    if (!p.filepath.empty()) {
      std::vector<float> h((size_t)m * (size_t)m);
      int64_t orig = 0;
      amm_compat::check(amm_read_matrix_file(p.filepath.c_str(), h.data(), (int64_t)m, &orig),
                        "amm_read_matrix_file");
      if (cudaMemcpy(dA, h.data(), sizeof(float) * h.size(), cudaMemcpyHostToDevice) !=
          cudaSuccess)
        throw amm_compat::error(AMM_ERR_CUDA, "write_data upload");
      p.diagonal_offset = 0.0f;
    } else {
      float off = 0.0f;
      amm_compat::check(amm_generate_matrix(p.matrixType.c_str(), (int64_t)m, seed, (float*)dA,
                                            &off, stream_1),
                        "amm_generate_matrix");
      p.diagonal_offset = off;
      gen_pos += m * m;
    }
    matrix_ready = true;
  }

  // As the reference's write_data (:316-337): A (loaded, generated, or the caller's when
  // matrix_ready is set) is bound and its column statistics and ||alpha||^2 are computed.
  void write_data(host_memory& p) {
    if (!matrix_ready) load_or_generate(p);
    amm_compat::check(amm_set_matrix(ctx, dA, (int64_t)m, stream_1), "amm_set_matrix");
    double a2 = 0.0;
    amm_compat::check(
        amm_get_column_stats(ctx, nullptr, nullptr, nullptr, nullptr, nullptr, &a2, stream_1),
        "amm_get_column_stats");
    p.alpha2 = (float)a2;
  }

  // xorshift states from -seed (:339-343), at the generator's current position.
  void set_internal_randomness() {
    const int64_t count = (int64_t)(m > c ? m : c);
    amm_compat::check(amm_seed_rng_at(ctx, seed, gen_pos, count, stream_1), "amm_seed_rng_at");
    gen_pos += (uint64_t)count;
  }

  // The start-vector generator, re-seeded like AMM.cu:85 (1234 + seed), continuing from the
  // position the states left it at.
  void seed_start_vectors(uint64_t s) {
    amm_compat::check(amm_seed_start_vectors_at(ctx, s, gen_pos), "amm_seed_start_vectors_at");
  }

  void zero_clear() { is_init = true; }
};

namespace amm_compat {

// One call plus the reference's reporting: (time_ms, eig, err) per step, eig =
// max(0, sqrt(max(0, λ)) − offset), err = 1 − e² (powerMethod_by_exact.cuh:74-93).
inline void run(host_memory& p, device_memory& dm, int method, bool is_output) {
  dm.zero_clear();
  check(amm_draw_start_vector(dm.ctx, dm.dx, dm.stream_1), "amm_draw_start_vector");
  check(amm_power_method(dm.ctx, method, dm.dx, dm.stream_1), "amm_power_method");
  std::vector<double> eigs(p.step), errs(p.step), t(p.step);
  int64_t run = 0;
  check(amm_get_trace(dm.ctx, eigs.data(), errs.data(), nullptr, nullptr, nullptr, t.data(), &run,
                      dm.stream_1),
        "amm_get_trace");
  if (!is_output) return;
  for (int64_t i = 0; i < run; ++i) {
    const double time = t[i] * 1e-6;
    const double eig = std::max(0.0, std::sqrt(std::max(0.0, eigs[i])) - p.diagonal_offset);
    const double err = 1.0 - errs[i] * errs[i];
    if (p.display) printf("%.12lf,%.12lf,%.12lf\n", time, eig, err);
    dm.ofs_output.write(reinterpret_cast<const char*>(&time), sizeof(double));
    dm.ofs_output.write(reinterpret_cast<const char*>(&eig), sizeof(double));
    dm.ofs_output.write(reinterpret_cast<const char*>(&err), sizeof(double));
  }
}

}  // namespace amm_compat

// powerMethod_by_exact.cuh:4-100
inline void powerMethod_by_exact(host_memory& p, device_memory& dm, const bool is_output = true) {
  amm_compat::run(p, dm, AMM_METHOD_EXACT, is_output);
}
// powerMethod_by_previous.cuh:100-210
inline void powerMethod_by_previous(host_memory& p, device_memory& dm, const bool is_output = true) {
  amm_compat::run(p, dm, AMM_METHOD_PREVIOUS, is_output);
}
// powerMethod_by_proposed.cuh:317-447
inline void powerMethod_by_proposed(host_memory& p, device_memory& dm, const bool is_output = true) {
  amm_compat::run(p, dm, AMM_METHOD_PROPOSED, is_output);
}
// powerMethod_by_proposed_v2.cuh:199-377
inline void powerMethod_by_proposed_v2(host_memory& p, device_memory& dm,
                                       const bool is_output = true) {
  amm_compat::run(p, dm, AMM_METHOD_PROPOSED_V2, is_output);
}

// square_of_A_by_previous / _proposed: one sampled product y = Ĉ·x on caller buffers
// (x, x_memo, y_memo in, y out; device pointers of length m).
inline void square_of_A_by_previous(device_memory& dm, const float* x, const float* x_memo,
                                    const float* y_memo, float* y) {
  amm_compat::check(amm_core_previousAMM(dm.ctx, x, x_memo, y_memo, y, nullptr, dm.stream_1),
                    "amm_core_previousAMM");
}
inline void square_of_A_by_proposed(device_memory& dm, const float* x, const float* x_memo,
                                    const float* y_memo, float* y) {
  amm_compat::check(amm_core_proposedAMM(dm.ctx, x, x_memo, y_memo, y, nullptr, dm.stream_1),
                    "amm_core_proposedAMM");
}

#endif  // AMM_COMPAT_HPP_
