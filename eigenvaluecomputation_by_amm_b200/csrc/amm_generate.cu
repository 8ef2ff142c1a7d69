// Matrix sources of the reference's driver: the on-device generators (-matrixType) and the
// covariance-file loader (-filepath), device_memory.h:360-433 and host_memory.h:143-159.
//
// Generators: a cuRAND XORWOW generator seeded with the run's seed fills the size x size matrix
// (column-major, ld = size) with N(p1, p2), lognormal(p1, p2) or U(p1, p2) values; the strictly
// lower triangle is mirrored into the upper one, and a diagonal offset derived from the row sums
// (a Gershgorin-style shift) is added so that the power method sees a PSD matrix.  The same
// cuRAND calls in the same order give the same matrix as the reference for the same seed.
//
// The offset: for each column i, max(0, Σ_r |a_ri| − 2·|a_ii|) summed sequentially in FP32;
// the reference takes the 1-based index of the largest of these from cublasIsamax and then
// reads the value one PAST it (device_memory.h:428-429).  That reading is reproduced here
// (the value after the largest, or the largest itself when it is the last column, where the
// reference reads past its buffer), so results match the reference's run for run.

#include <cuda_runtime.h>
#include <curand.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "amm.h"
#include "amm_internal.h"

namespace amm {
namespace {

__global__ void shift_scale_kernel(float* d, uint64_t len, float a, float b) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < len;
       i += (uint64_t)gridDim.x * blockDim.x)
    d[i] = fmaf(b - a, d[i], a);  // a + (b − a)·u, one rounding as the contracted reference
}

// (row x, column y) of the upper triangle <- (row y, column x) of the lower one
__global__ void mirror_kernel(float* d, uint64_t size) {
  const uint64_t len = size * size;
  for (uint64_t idx = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; idx < len;
       idx += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t y = idx % size, x = idx / size;
    if (x < y) d[x + y * size] = d[idx];
  }
}

__global__ void row_excess_kernel(float* out, const float* d, uint64_t size) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= size) return;
  const float* col = d + size * i;
  float s = 0.0f;
  for (uint64_t r = 0; r < size; ++r) s += fabsf(col[r]);
  out[i] = fmaxf(0.0f, fmaf(-2.0f, fabsf(d[i + i * size]), s));
}

// The offset as the reference reads it (see the file comment), one thread.
__global__ void pick_offset_kernel(const float* ex, uint64_t size, float* offset) {
  uint64_t best = 0;
  float bv = fabsf(ex[0]);
  for (uint64_t i = 1; i < size; ++i) {
    const float v = fabsf(ex[i]);
    if (v > bv) {
      bv = v;
      best = i;
    }
  }
  *offset = ex[best + 1 < size ? best + 1 : best];
}

__global__ void add_diag_kernel(float* d, uint64_t size, const float* offset) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i < size) d[i + i * size] += *offset;
}

std::vector<std::string> split(const std::string& s, char sep) {
  std::vector<std::string> v;
  size_t b = 0;
  for (;;) {
    const size_t e = s.find(sep, b);
    v.push_back(s.substr(b, e == std::string::npos ? std::string::npos : e - b));
    if (e == std::string::npos) break;
    b = e + 1;
  }
  return v;
}

}  // namespace
}  // namespace amm

extern "C" int amm_generate_matrix(const char* type, int64_t size, uint64_t seed, float* d_A,
                                   float* offset_out, void* stream) {
  if (!type || !d_A || size < 1 || (size * size) % 2 != 0) return AMM_ERR_INVALID_ARGUMENT;
  // "<kind>_<p1>_<p2>" (extract_parames, device_memory.h:487-497)
  const auto ary = amm::split(type, '_');
  const std::string kind = ary[0];
  const float p1 = ary.size() <= 1 ? 0.0f : (float)std::atof(ary[1].c_str());
  const float p2 = ary.size() <= 2 ? 0.0f : (float)std::atof(ary[2].c_str());
  if (kind != "gaussian" && kind != "lognormal" && kind != "uniform") return AMM_ERR_UNSUPPORTED;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const uint64_t n = (uint64_t)size, len = n * n;
  curandGenerator_t gen;
  if (curandCreateGenerator(&gen, CURAND_RNG_PSEUDO_DEFAULT) != CURAND_STATUS_SUCCESS)
    return AMM_ERR_CUDA;
  curandStatus_t cs = curandSetStream(gen, s);
  if (cs == CURAND_STATUS_SUCCESS) cs = curandSetPseudoRandomGeneratorSeed(gen, seed);
  if (cs == CURAND_STATUS_SUCCESS) {
    if (kind == "gaussian")
      cs = curandGenerateNormal(gen, d_A, len, p1, p2);
    else if (kind == "lognormal")
      cs = curandGenerateLogNormal(gen, d_A, len, p1, p2);
    else
      cs = curandGenerateUniform(gen, d_A, len);
  }
  curandDestroyGenerator(gen);
  if (cs != CURAND_STATUS_SUCCESS) return AMM_ERR_CUDA;
  float* work = nullptr;  // size excess values + the offset
  cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&work), sizeof(float) * (n + 1), s);
  if (e != cudaSuccess) return amm::record_cuda_failure(e, "cudaMallocAsync");
  const int T = 256;
  const int blocks = (int)std::min<uint64_t>((len + T - 1) / T, 65535ull * 16);
  if (kind == "uniform") amm::shift_scale_kernel<<<blocks, T, 0, s>>>(d_A, len, p1, p2);
  amm::mirror_kernel<<<blocks, T, 0, s>>>(d_A, n);
  amm::row_excess_kernel<<<(int)((n + 127) / 128), 128, 0, s>>>(work, d_A, n);
  amm::pick_offset_kernel<<<1, 1, 0, s>>>(work, n, work + n);
  amm::add_diag_kernel<<<(int)((n + 127) / 128), 128, 0, s>>>(d_A, n, work + n);
  amm::count_launch(kind == "uniform" ? 5 : 4);
  float off = 0.0f;
  e = cudaMemcpyAsync(&off, work + n, sizeof(float), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaFreeAsync(work, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return amm::record_cuda_failure(e, "amm_generate_matrix");
  if (offset_out) *offset_out = off;
  return AMM_OK;
}

extern "C" int amm_read_matrix_file(const char* path, float* h_A, int64_t size,
                                    int64_t* original_size) {
  if (!path) return AMM_ERR_INVALID_ARGUMENT;
  std::ifstream ifs(path, std::ios::in | std::ios::binary);
  if (!ifs.good()) return AMM_ERR_INVALID_ARGUMENT;
  uint32_t orig = 0;
  ifs.read(reinterpret_cast<char*>(&orig), sizeof(uint32_t));
  if (!ifs.good() || orig == 0) return AMM_ERR_INVALID_ARGUMENT;
  if (original_size) *original_size = orig;
  if (!h_A) return AMM_OK;  // size query only
  if (size < (int64_t)orig) return AMM_ERR_INVALID_ARGUMENT;
  std::memset(h_A, 0, sizeof(float) * (size_t)size * (size_t)size);
  std::vector<float> row(orig);
  for (uint32_t y = 0; y < orig; ++y) {  // file row y -> h_A[y*size + x]
    ifs.read(reinterpret_cast<char*>(row.data()), sizeof(float) * orig);
    if (!ifs.good()) return AMM_ERR_INVALID_ARGUMENT;
    std::memcpy(h_A + (size_t)y * (size_t)size, row.data(), sizeof(float) * orig);
  }
  return AMM_OK;
}
