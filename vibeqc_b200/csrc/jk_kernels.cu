// Coulomb build J[mu][nu] = sum_Q B[mu][Q][nu] rho[Q] over the FP32 whitened
// tensor stored aux-major per AO row, B[mol][mu][Q][nu] (row length ld >= N).
// Reference: src/scf/cuda/df_coulomb.cpp:24 (packed cublasDgemv, FP64).
//
// HBM-streaming: one CTA per (molecule, mu) reads only the nu <= mu half of
// B[mu] (J is symmetric), coalesced along nu, accumulates in FP64 with rho
// staged in shared memory, and writes J[mu][nu] and its mirror J[nu][mu].
#include "vqc_df.h"
#include "vqc_plan.hpp"

namespace vqc {

constexpr int kJThreads = 128;
constexpr int kJMaxNu = 4;  // nu per thread: N <= 512

__global__ void __launch_bounds__(kJThreads)
    coulomb_fp32_kernel(const float* __restrict__ b, const double* __restrict__ rho, int n, int x,
                        int ld, double* __restrict__ j) {
  extern __shared__ double srho[];
  const int mol = blockIdx.y, mu = blockIdx.x;
  for (int q = threadIdx.x; q < x; q += kJThreads) srho[q] = rho[(size_t)mol * x + q];
  __syncthreads();
  const float* row = b + ((size_t)mol * n + mu) * (size_t)x * ld;
  double acc[kJMaxNu];
#pragma unroll
  for (int t = 0; t < kJMaxNu; ++t) acc[t] = 0.0;
  const int nu_end = mu + 1;  // lower triangle nu <= mu
  int q = 0;
  for (; q + 4 <= x; q += 4) {
    const double r0 = srho[q], r1 = srho[q + 1], r2 = srho[q + 2], r3 = srho[q + 3];
    const float* p0 = row + (size_t)q * ld;
#pragma unroll
    for (int t = 0; t < kJMaxNu; ++t) {
      const int nu = threadIdx.x + t * kJThreads;
      if (nu < nu_end) {
        const float v0 = __ldg(p0 + nu), v1 = __ldg(p0 + ld + nu), v2 = __ldg(p0 + 2 * ld + nu),
                    v3 = __ldg(p0 + 3 * ld + nu);
        acc[t] = fma((double)v0, r0, acc[t]);
        acc[t] = fma((double)v1, r1, acc[t]);
        acc[t] = fma((double)v2, r2, acc[t]);
        acc[t] = fma((double)v3, r3, acc[t]);
      }
    }
  }
  for (; q < x; ++q) {
    const double r = srho[q];
#pragma unroll
    for (int t = 0; t < kJMaxNu; ++t) {
      const int nu = threadIdx.x + t * kJThreads;
      if (nu < nu_end) acc[t] = fma((double)__ldg(row + (size_t)q * ld + nu), r, acc[t]);
    }
  }
  double* jm = j + (size_t)mol * n * n;
#pragma unroll
  for (int t = 0; t < kJMaxNu; ++t) {
    const int nu = threadIdx.x + t * kJThreads;
    if (nu < nu_end) {
      jm[(size_t)mu * n + nu] = acc[t];
      jm[(size_t)nu * n + mu] = acc[t];
    }
  }
}

// B[mol][mu][Q][nu] (FP32, ld) from the whitened packed rows
// bp[mol][(max(mu,nu)(max+1)/2 + min)][Q] (FP64); padding columns are zeroed.
__global__ void __launch_bounds__(256)
    unpack_aux_major_kernel(const double* __restrict__ bp, int n, int x, int ld,
                            float* __restrict__ b) {
  const int mol = blockIdx.z, mu = blockIdx.y;
  const size_t p = (size_t)n * (n + 1) / 2;
  const double* src = bp + (size_t)mol * p * x;
  float* dst = b + ((size_t)mol * n + mu) * (size_t)x * ld;
  // tile over (Q, nu): threads run along nu for coalesced stores
  const size_t total = (size_t)x * ld;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (size_t)gridDim.x * blockDim.x) {
    const int q = (int)(e / ld), nu = (int)(e % ld);
    float v = 0.0f;
    if (nu < n) {
      const size_t hi = mu > nu ? mu : nu, lo = mu > nu ? nu : mu;
      v = (float)src[(hi * (hi + 1) / 2 + lo) * x + q];
    }
    dst[e] = v;
  }
}

}  // namespace vqc

using namespace vqc;

extern "C" int vqc_coulomb_fp32(const float* b_aux_major, const double* rho, int32_t nmol,
                                int32_t nao, int32_t ld_ao, int32_t naux, double* j, void* stream) {
  if (!b_aux_major || !rho || !j || nmol <= 0 || nao <= 0 || naux <= 0 || ld_ao < nao ||
      nao > kJThreads * kJMaxNu || nmol > 65535)
    return fail(VQC_STATUS_INVALID_ARGUMENT, "coulomb_fp32: bad argument");
  const size_t smem = (size_t)naux * sizeof(double);
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(coulomb_fp32_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_status(e, "coulomb_fp32 smem");
  }
  dim3 grid(nao, nmol);
  coulomb_fp32_kernel<<<grid, kJThreads, smem, (cudaStream_t)stream>>>(b_aux_major, rho, nao, naux,
                                                                        ld_ao, j);
  count_launch();
  return cuda_status(cudaGetLastError(), "coulomb_fp32");
}

extern "C" int vqc_unpack_aux_major(const double* b_packed, int32_t nmol, int32_t nao, int32_t naux,
                                    int32_t ld_ao, float* b_aux_major, void* stream) {
  if (!b_packed || !b_aux_major || nmol <= 0 || nao <= 0 || naux <= 0 || ld_ao < nao ||
      nmol > 65535 || nao > 65535)
    return fail(VQC_STATUS_INVALID_ARGUMENT, "unpack_aux_major: bad argument");
  const size_t per = (size_t)naux * ld_ao;
  int bx = (int)((per + 255) / 256);
  bx = bx > 64 ? 64 : bx;
  dim3 grid(bx, nao, nmol);
  unpack_aux_major_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(b_packed, nao, naux, ld_ao,
                                                                  b_aux_major);
  count_launch();
  return cuda_status(cudaGetLastError(), "unpack_aux_major");
}
