// Launch-side definitions shared by the kernel translation units and the
// plan/C-ABI layer.
#pragma once

#include "vqc_internal.cuh"

namespace vqc {

// per (angular-momentum class, molecule) work entry
struct ClassMol {
  int mol;
  int pair_begin;   // first pair of this molecule in the class pair list
  int aux_begin;    // first aux shell with the class aux l in this molecule
  int naux;         // number of such aux shells
  int ntriples;     // work items (pairs x aux shells, or pairs)
  int chunk_begin;  // first CTA of this entry
};

struct ClassLaunch {
  int la, lb, lc;
  const int2* pairs;
  const ClassMol* cms;
  int ncm;
  int nblocks;
};

struct KernelArgs {
  DevBasis orb, aux;
  const double* xyz;
  const double* charge;
  const DevMol* mols;
  double* out;
  double* out2;
  double* out3;
  const double* w1;  // derivative weights (Abar / Mbar / densities)
  const double* w2;
  double* grad;
};

__host__ __device__ constexpr int out_count(int l, bool sph) { return sph ? 2 * l + 1 : (l + 1) * (l + 2) / 2; }

// triples per CTA of the 3-centre value kernel: <= 256 threads and a shared
// staging block of at most 40 KB
__host__ __device__ constexpr int slots3c(int la, int lb, int lc, bool sph) {
  return (256 / ncart(lc)) < (5120 / (ncart(lc) * out_count(la, sph) * out_count(lb, sph)))
             ? (256 / ncart(lc))
             : (5120 / (ncart(lc) * out_count(la, sph) * out_count(lb, sph)));
}

// Resident CTAs per SM requested from the compiler for the 3-centre kernels:
// the low-l classes (the most frequent and the most contracted) are latency-
// bound on FP64 dependencies at one or two CTAs, so they are compiled to fit
// more (fewer registers, a few hundred bytes of spills); the high-l classes
// keep their registers.  Measured on 48 clusters: values 127 -> 79 ms,
// derivatives 171 -> 128 ms per step.
__host__ __device__ constexpr int min_ctas3c(int la, int lb, int lc) {
  return la + lb + lc <= 3 ? 3 : (la + lb + lc <= 5 ? 2 : 1);
}
__host__ __device__ constexpr int min_ctas_grad3c(int la, int lb, int lc) {
  return la + lb + lc <= 5 ? 2 : 1;
}
// Resident CTAs per SM requested for the root-parallel 3-centre kernels:
// enough for about 512 threads per SM (at most 128 registers a thread).
__host__ __device__ constexpr int min_ctas_rp(int threads) {
  return threads >= 512 ? 1 : (512 / threads > 8 ? 8 : 512 / threads);
}

template <int LA, int LB, int LC, bool SPH>
struct Int3cCfg {
  static constexpr int NOA = out_count(LA, SPH), NOB = out_count(LB, SPH), NOC = out_count(LC, SPH);
  static constexpr int SLOTS = slots3c(LA, LB, LC, SPH);
  static constexpr int THREADS = SLOTS * ncart(LC);
};

__host__ __device__ constexpr int slots2c(int lc) { return 256 / ncart(lc); }

template <int LA, int LC, bool SPH>
struct Int2cCfg {
  static constexpr int NOA = out_count(LA, SPH), NOC = out_count(LC, SPH);
  static constexpr int SLOTS = slots2c(LC);
  static constexpr int THREADS = SLOTS * ncart(LC);
};

bool dispatch_int3c(const ClassLaunch& cl, const KernelArgs& k, bool sph, cudaStream_t st);
bool dispatch_int2c(const ClassLaunch& cl, const KernelArgs& k, bool sph, cudaStream_t st);
bool dispatch_int1e(const ClassLaunch& cl, const KernelArgs& k, bool sph, cudaStream_t st);
bool dispatch_grad3c(const ClassLaunch& cl, const KernelArgs& k, bool sph, cudaStream_t st);
bool dispatch_grad2c(const ClassLaunch& cl, const KernelArgs& k, bool sph, cudaStream_t st);
bool dispatch_grad1e(const ClassLaunch& cl, const KernelArgs& k, bool sph, cudaStream_t st);

}  // namespace vqc
