// Coulomb build J[mu][nu] = sum_Q B[mu][Q][nu] rho[Q] over the FP32 whitened
// tensor stored aux-major per AO row, B[mol][mu][Q][nu] (row length ld >= N).
// Reference: src/scf/cuda/df_coulomb.cpp:24 (packed cublasDgemv, FP64).
//
// HBM-streaming: one CTA per (molecule, mu) reads only the nu <= mu half of
// B[mu] (J is symmetric).  A row holds nvec = ceil((mu + 1) / 4) float4; each
// warp splits into groups of L = min(32, pow2 >= nvec) lanes so short rows do
// not idle lanes, and every group streams kJRows independent Q rows per pass
// (memory-level parallelism).  Accumulation is FP64 with rho staged in shared
// memory; group and warp partials are summed through shuffles and shared
// memory into J[mu][nu] and J[nu][mu].
#include <mutex>

#include "vqc_df.h"
#include "vqc_plan.hpp"

namespace vqc {

constexpr int kJThreads = 256;          // 8 warps share the Q range of one (mol, mu) row
constexpr int kJWarps = kJThreads / 32;
constexpr int kJMaxVec = 4;             // float4 per lane: nu < 4 * 32 * 4 = 512
constexpr int kJRows = 4;               // Q rows per lane group per pass

__device__ __forceinline__ int group_lanes(int nvec) {
  int l = 1;
  while (l < nvec && l < 32) l <<= 1;
  return l;
}

// MV = float4 columns per lane (rows up to 128 * MV): the accumulators scale
// with the row length, so short rows keep registers (and occupancy) low
template <int MV>
__global__ void __launch_bounds__(kJThreads)
    coulomb_fp32_kernel(const float* __restrict__ b, const double* __restrict__ rho, int n, int x,
                        int ld, double* __restrict__ j) {
  extern __shared__ double smem[];
  double* srho = smem;                          // x
  double* part = smem + ((x + 1) & ~1);         // kJWarps * ld partial sums
  const int mol = blockIdx.y, mu = blockIdx.x;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int q = threadIdx.x; q < x; q += kJThreads) srho[q] = rho[(size_t)mol * x + q];
  __syncthreads();
  const float* rowb = b + ((size_t)mol * n + mu) * (size_t)x * ld;
  const int nvec = (mu + 1 + 3) / 4;  // float4 columns covering nu <= mu (ld % 4 == 0)
  const int L = group_lanes(nvec), G = 32 / L, grp = lane / L, gl = lane % L;
  const int rstride = kJWarps * G;  // lane groups per CTA
  double acc[MV][4];
#pragma unroll
  for (int t = 0; t < MV; ++t)
#pragma unroll
    for (int e = 0; e < 4; ++e) acc[t][e] = 0.0;
  // q0 - grp is the same for every lane of the warp: the trip count is uniform
  for (int q0 = warp * G + grp; q0 - grp < x; q0 += kJRows * rstride) {
#pragma unroll
    for (int t = 0; t < MV; ++t) {
      const int v = gl + L * t;
      if (v < nvec) {
        float4 f[kJRows];
        double r[kJRows];
#pragma unroll
        for (int k = 0; k < kJRows; ++k) {
          const int q = q0 + k * rstride;
          const bool ok = q < x;
          r[k] = ok ? srho[q] : 0.0;
          f[k] = ok ? __ldg(reinterpret_cast<const float4*>(rowb + (size_t)q * ld) + v)
                    : make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
        for (int k = 0; k < kJRows; ++k) {
          acc[t][0] = fma((double)f[k].x, r[k], acc[t][0]);
          acc[t][1] = fma((double)f[k].y, r[k], acc[t][1]);
          acc[t][2] = fma((double)f[k].z, r[k], acc[t][2]);
          acc[t][3] = fma((double)f[k].w, r[k], acc[t][3]);
        }
      }
    }
  }
  // sum the lane groups of the warp (lanes with equal gl)
  for (int off = L; off < 32; off <<= 1)
#pragma unroll
    for (int t = 0; t < MV; ++t)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[t][e] += __shfl_xor_sync(0xffffffffu, acc[t][e], off);
  if (grp == 0) {
#pragma unroll
    for (int t = 0; t < MV; ++t) {
      const int v = gl + L * t;
      if (v < nvec) {
#pragma unroll
        for (int e = 0; e < 4; ++e) part[warp * ld + 4 * v + e] = acc[t][e];
      }
    }
  }
  __syncthreads();
  double* jm = j + (size_t)mol * n * n;
  for (int nu = threadIdx.x; nu <= mu; nu += kJThreads) {
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < kJWarps; ++w) s += part[w * ld + nu];
    jm[(size_t)mu * n + nu] = s;
    jm[(size_t)nu * n + mu] = s;
  }
}

// Fitted density rho[mol][Q] = sum_{mu,nu} B[mu][Q][nu] D[mu][nu] (D symmetric),
// read from the nu <= mu half with weights 2 (nu < mu) and 1 (nu = mu).
// Stage 1: one CTA per (molecule, mu), shaped like the Coulomb kernel (lane
// groups sized to the row, kJRows independent Q rows per group and pass,
// weighted density row staged in shared memory), writes the row partial
// part[mol][mu][Q] (FP64, shuffle sums within the group).  Stage 2 adds the
// partials over mu in a fixed order, so the result is deterministic.
// Reference: rho = B^T vec(D) of src/scf/cuda/df_coulomb.cpp:38-57 (FP64
// cublasDgemv).
template <int MV>
__global__ void __launch_bounds__(kJThreads)
    fitted_rows_fp32_kernel(const float* __restrict__ b, const double* __restrict__ d, int n,
                            int x, int ld, double* __restrict__ part) {
  extern __shared__ double sw[];  // weighted density row, ld entries
  const int mol = blockIdx.y, mu = blockIdx.x;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const double* drow = d + ((size_t)mol * n + mu) * n;
  for (int nu = threadIdx.x; nu < ld; nu += kJThreads)
    sw[nu] = nu < mu ? 2.0 * drow[nu] : (nu == mu ? drow[nu] : 0.0);
  __syncthreads();
  const float* rowb = b + ((size_t)mol * n + mu) * (size_t)x * ld;
  const int nvec = (mu + 1 + 3) / 4;
  const int L = group_lanes(nvec), G = 32 / L, grp = lane / L, gl = lane % L;
  const int rstride = kJWarps * G;
  double* out = part + ((size_t)mol * n + mu) * x;
  for (int q0 = warp * G + grp; q0 - grp < x; q0 += kJRows * rstride) {  // warp-uniform trips
    double acc[kJRows];
#pragma unroll
    for (int k = 0; k < kJRows; ++k) acc[k] = 0.0;
#pragma unroll
    for (int t = 0; t < MV; ++t) {
      const int v = gl + L * t;
      if (v < nvec) {
        const double w0 = sw[4 * v], w1 = sw[4 * v + 1], w2 = sw[4 * v + 2], w3 = sw[4 * v + 3];
        float4 f[kJRows];
#pragma unroll
        for (int k = 0; k < kJRows; ++k) {
          const int q = q0 + k * rstride;
          f[k] = q < x ? __ldg(reinterpret_cast<const float4*>(rowb + (size_t)q * ld) + v)
                       : make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
        for (int k = 0; k < kJRows; ++k) {
          acc[k] = fma((double)f[k].x, w0, acc[k]);
          acc[k] = fma((double)f[k].y, w1, acc[k]);
          acc[k] = fma((double)f[k].z, w2, acc[k]);
          acc[k] = fma((double)f[k].w, w3, acc[k]);
        }
      }
    }
#pragma unroll
    for (int k = 0; k < kJRows; ++k) {
      double sum = acc[k];
      for (int off = L >> 1; off > 0; off >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, off, L);
      const int q = q0 + k * rstride;
      if (gl == 0 && q < x) out[q] = sum;
    }
  }
}

__global__ void __launch_bounds__(256)
    fitted_sum_kernel(const double* __restrict__ part, int n, int x, double* __restrict__ rho) {
  const int mol = blockIdx.y;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= x) return;
  const double* p = part + (size_t)mol * n * x + q;
  double s = 0.0;
  for (int mu = 0; mu < n; ++mu) s += p[(size_t)mu * x];
  rho[(size_t)mol * x + q] = s;
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

// Incremental exchange about an FP64 anchor U0 = B C0 ([row][Q], rows of
// length x) and the tensor-core increment dU = B (C - C0) (split hi/lo, rows
// of length ldq):
//   mode 0: V = U0 + alpha (dU_hi + dU_lo), written split into v_hi / v_lo
//           (round-to-nearest TF32 parts, padding columns zero);
//   mode 1: U0 += alpha (dU_hi + dU_lo) in place (FP64).
__global__ void __launch_bounds__(256)
    anchor_combine_kernel(double* __restrict__ u0, const float* __restrict__ du_hi,
                          const float* __restrict__ du_lo, float* __restrict__ v_hi,
                          float* __restrict__ v_lo, long long rows, int x, int ldq, double alpha,
                          int mode) {
  const long long total = rows * (long long)ldq;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long r = e / ldq;
    const int q = (int)(e - r * ldq);
    if (q >= x) {
      if (mode == 0) {
        v_hi[e] = 0.0f;
        v_lo[e] = 0.0f;
      }
      continue;
    }
    const double d = (double)__ldg(du_hi + e) + (double)__ldg(du_lo + e);
    double* p = u0 + r * x + q;
    if (mode == 1) {
      *p += alpha * d;
    } else {
      const float v = (float)(*p + alpha * d);
      uint32_t hb, lb;
      asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(hb) : "f"(v));
      const float h = __uint_as_float(hb);
      asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(lb) : "f"(v - h));
      v_hi[e] = h;
      v_lo[e] = __uint_as_float(lb);
    }
  }
}

}  // namespace vqc

using namespace vqc;

extern "C" int vqc_anchor_combine(double* u0, const float* du_hi, const float* du_lo, float* v_hi,
                                  float* v_lo, int64_t rows, int32_t x, int32_t ld_aux,
                                  double alpha, int32_t mode, void* stream) {
  if (!u0 || !du_hi || !du_lo || rows <= 0 || x <= 0 || ld_aux < x || (mode != 0 && mode != 1) ||
      (mode == 0 && (!v_hi || !v_lo)))
    return fail(VQC_STATUS_INVALID_ARGUMENT, "anchor_combine: bad argument");
  long long blocks = (rows * (long long)ld_aux + 255) / 256;
  blocks = blocks > 8 * 148 ? 8 * 148 : blocks;
  anchor_combine_kernel<<<(int)blocks, 256, 0, (cudaStream_t)stream>>>(
      u0, du_hi, du_lo, v_hi, v_lo, (long long)rows, x, ld_aux, alpha, mode);
  count_launch();
  return cuda_status(cudaGetLastError(), "anchor_combine");
}

extern "C" int vqc_coulomb_fp32(const float* b_aux_major, const double* rho, int32_t nmol,
                                int32_t nao, int32_t ld_ao, int32_t naux, double* j, void* stream) {
  if (!b_aux_major || !rho || !j || nmol <= 0 || nao <= 0 || naux <= 0 || ld_ao < nao ||
      ld_ao % 4 || ld_ao > 4 * 32 * kJMaxVec || nmol > 65535 || nao > 65535)
    return fail(VQC_STATUS_INVALID_ARGUMENT, "coulomb_fp32: bad argument");
  const size_t smem = ((size_t)((naux + 1) & ~1) + (size_t)kJWarps * ld_ao) * sizeof(double);
  if (smem > 200 * 1024) return fail(VQC_STATUS_INVALID_ARGUMENT, "coulomb_fp32: too many auxiliary functions");
  dim3 grid(nao, nmol);
  const int mv = (ld_ao / 4 + 31) / 32;
  auto kern = mv <= 1 ? coulomb_fp32_kernel<1>
              : mv == 2 ? coulomb_fp32_kernel<2>
              : mv == 3 ? coulomb_fp32_kernel<3>
                        : coulomb_fp32_kernel<4>;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_status(e, "coulomb_fp32 smem");
  }
  kern<<<grid, kJThreads, smem, (cudaStream_t)stream>>>(b_aux_major, rho, nao, naux, ld_ao, j);
  count_launch();
  return cuda_status(cudaGetLastError(), "coulomb_fp32");
}

extern "C" int vqc_fitted_density_fp32(const float* b_aux_major, const double* dens, int32_t nmol,
                                       int32_t nao, int32_t ld_ao, int32_t naux, double* partial,
                                       double* rho, void* stream) {
  if (!b_aux_major || !dens || !partial || !rho || nmol <= 0 || nao <= 0 || naux <= 0 ||
      ld_ao < nao || ld_ao % 4 || ld_ao > 4 * 32 * kJMaxVec || nmol > 65535)
    return fail(VQC_STATUS_INVALID_ARGUMENT, "fitted_density_fp32: bad argument");
  const size_t smem = (size_t)ld_ao * sizeof(double);
  if (smem > 48 * 1024) return fail(VQC_STATUS_INVALID_ARGUMENT, "fitted_density_fp32: nao too large");
  dim3 g1(nao, nmol);
  const int mv = (ld_ao / 4 + 31) / 32;
  auto kern = mv <= 1 ? fitted_rows_fp32_kernel<1>
              : mv == 2 ? fitted_rows_fp32_kernel<2>
              : mv == 3 ? fitted_rows_fp32_kernel<3>
                        : fitted_rows_fp32_kernel<4>;
  kern<<<g1, kJThreads, smem, (cudaStream_t)stream>>>(b_aux_major, dens, nao, naux, ld_ao, partial);
  count_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_status(e, "fitted_density_fp32 rows");
  dim3 g2((naux + 255) / 256, nmol);
  fitted_sum_kernel<<<g2, 256, 0, (cudaStream_t)stream>>>(partial, nao, naux, rho);
  count_launch();
  return cuda_status(cudaGetLastError(), "fitted_density_fp32 sum");
}

// No-allocation variant of vqc_fitted_density_fp32, for callers that cannot
// allocate device memory: a host program whose GPU memory is already owned by
// another allocator's pool (a framework's caching allocator, a fixed arena),
// or one that must not pay the device-wide synchronisation cudaFree implies.
// The per-row partial sums live in a file-scope device array of fixed
// capacity instead of a caller-owned buffer; every GPU that loads the library
// holds it until the process exits.  The first call on a device takes the
// array's device address with cudaGetSymbolAddress (that device current) and
// caches it, so that first call should come before any stream capture.
// Every call shares the array, which keeps the last call's contents; nothing
// in it must start at zero, because stage 1 writes every partial that the
// same launch's stage 2 reads.  Calls that overlap on the GPU race.
constexpr size_t kFittedScratchDoubles = (size_t)1 << 22;  // 32 MiB
static __device__ __align__(256) double g_fitted_scratch[kFittedScratchDoubles];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_scratch_mutex;
double* g_scratch_ptr[kMaxDevices] = {};
}  // namespace

static int fitted_scratch(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_status(e, "fitted_density_fp32_noalloc: device");
  if (dev < 0 || dev >= kMaxDevices)
    return fail(VQC_STATUS_INVALID_ARGUMENT, "fitted_density_fp32_noalloc: device index out of range");
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_fitted_scratch);
    if (e != cudaSuccess) return cuda_status(e, "fitted_density_fp32_noalloc: scratch address");
    g_scratch_ptr[dev] = static_cast<double*>(p);
  }
  *out = g_scratch_ptr[dev];
  return VQC_STATUS_SUCCESS;
}

extern "C" int vqc_fitted_density_fp32_noalloc(const float* b_aux_major, const double* dens,
                                               int32_t nmol, int32_t nao, int32_t ld_ao,
                                               int32_t naux, double* rho, void* stream) {
  if (!b_aux_major || !dens || !rho || nmol <= 0 || nao <= 0 || naux <= 0)
    return fail(VQC_STATUS_INVALID_ARGUMENT, "fitted_density_fp32_noalloc: bad argument");
  const size_t need = (size_t)nmol * (size_t)nao * (size_t)naux;
  if (need > kFittedScratchDoubles)
    return fail(VQC_STATUS_INVALID_ARGUMENT,
                "fitted_density_fp32_noalloc: nmol * nao * naux exceeds the 4194304-double scratch");
  double* part = nullptr;
  const int st = fitted_scratch(&part);
  if (st) return st;
  return vqc_fitted_density_fp32(b_aux_major, dens, nmol, nao, ld_ao, naux, part, rho, stream);
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
