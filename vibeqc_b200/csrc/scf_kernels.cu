// SCF-stage kernels over a batch of equally sized molecules.
//
// sp2_update: one step of second-order spectral projection (Niklasson,
// Phys. Rev. B 66, 155115 (2002)) for every molecule of a chunk, given
// X and X2 = X X (a batched GEMM).  Each CTA recomputes tr X and tr X^2 of its
// molecule, chooses X^2 or 2X - X^2 (whichever moves tr X toward n_occ) and
// writes its slice of the next iterate to a separate buffer.  A molecule whose
// idempotency error |tr X - tr X^2| fell below tol is copied unchanged and
// flagged, so a fixed number of steps can run without host synchronisation.  Replaces the per-iteration
// batched eigensolver of the reference's device SCF loop
// (src/scf/cuda/df_scf_library.cpp, cusolverDnXsyevBatched) for the density
// update.
#include "vqc_df.h"
#include "vqc_kernels.cuh"
#include "vqc_plan.hpp"

namespace vqc {

__device__ __forceinline__ double block_sum(double v, double* red) {
  for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x + 31) / 32 ? red[threadIdx.x] : 0.0;
    for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
    if (threadIdx.x == 0) red[0] = s;
  }
  __syncthreads();
  return red[0];
}

__global__ void __launch_bounds__(256) sp2_update_kernel(const double* __restrict__ x,
                                                         const double* __restrict__ x2,
                                                         double* __restrict__ xout, int n,
                                                         double nocc, double tol,
                                                         int* __restrict__ done) {
  __shared__ double red[32];
  const int m = blockIdx.y;
  const size_t base = (size_t)m * n * n;
  const size_t nn = (size_t)n * n;
  double t1 = 0.0, t2 = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    t1 += x[base + (size_t)i * n + i];
    t2 += x2[base + (size_t)i * n + i];
  }
  // inputs are never written by this kernel, so every CTA of a molecule sees
  // the same traces and takes the same branch
  const double tr = block_sum(t1, red);
  const double tr2 = block_sum(t2, red);
  const bool converged = done[m] != 0 || fabs(tr - tr2) < tol;
  const bool square = fabs(tr2 - nocc) < fabs(2.0 * tr - tr2 - nocc);
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < nn;
       idx += (size_t)gridDim.x * blockDim.x) {
    const double a = x[base + idx], b = x2[base + idx];
    xout[base + idx] = converged ? a : (square ? b : 2.0 * a - b);
  }
  if (converged && blockIdx.x == 0 && threadIdx.x == 0) done[m] = 1;
}

}  // namespace vqc

extern "C" int vqc_sp2_update(const double* x, const double* x2, double* xout, int32_t nmol,
                              int32_t n, double nocc, double tol, int32_t* done, void* stream) {
  using namespace vqc;
  if (!x || !x2 || !xout || !done || nmol <= 0 || n <= 0)
    return fail(VQC_STATUS_INVALID_ARGUMENT, "sp2_update: bad argument");
  const size_t nn = (size_t)n * n;
  int ctas = (int)((nn + 255 * 8 - 1) / (256 * 8));  // ~8 elements per thread
  ctas = ctas < 1 ? 1 : (ctas > 64 ? 64 : ctas);
  dim3 grid(ctas, nmol);
  sp2_update_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(x, x2, xout, n, nocc, tol, done);
  count_launch();
  return cuda_status(cudaGetLastError(), "sp2_update");
}
