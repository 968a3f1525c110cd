// Integral value kernels: one-electron S/T/V, 2-centre metric (P|Q) and
// 3-centre (mu nu|P), all FP64, for every angular-momentum class up to f.
//
// Work decomposition (3-centre): one thread per (orbital shell pair, aux shell,
// Cartesian aux component).  Each thread contracts its primitives, applies the
// orbital spherical transforms in registers and stages the block in shared
// memory; the CTA then applies the aux transform and writes rows of the
// packed tensor A[(mu nu)][P] so that consecutive threads store consecutive P.
//
// Reference behaviour: src/integrals/s_integrals.cpp:1201 (raw DF integrals),
// :1520 (spherical transform), :1865 (one-electron); CUDA counterpart
// src/scf/cuda/df_source_kernels.cu:67.
#include "vqc_kernels.cuh"

namespace vqc {

// ---------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------

__device__ __forceinline__ void cart_of(int l, int k, int& x, int& y, int& z) {
  int rem = k, lx = l;
  while (rem > l - lx) {
    rem -= l - lx + 1;
    --lx;
  }
  x = lx;
  y = l - lx - rem;
  z = rem;
}

// chunk -> class-molecule entry by binary search over chunk_begin
__device__ __forceinline__ int find_cm(const ClassMol* __restrict__ cms, int ncm, int block) {
  int lo = 0, hi = ncm - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (cms[mid].chunk_begin <= block) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// transform an (NCA x NCB) Cartesian block with the a/b output transforms
template <int LA, int LB, int NOA, int NOB>
__device__ __forceinline__ void transform_ab(int mode, const double (&acc)[ncart(LA)][ncart(LB)],
                                             double (&w)[NOA][NOB]) {
  double tmp[NOA][ncart(LB)];
#pragma unroll
  for (int i = 0; i < NOA; ++i)
#pragma unroll
    for (int y = 0; y < ncart(LB); ++y) {
      double s = 0.0;
#pragma unroll
      for (int x = 0; x < ncart(LA); ++x) s = fma(c_trans[mode][LA][i][x], acc[x][y], s);
      tmp[i][y] = s;
    }
#pragma unroll
  for (int i = 0; i < NOA; ++i)
#pragma unroll
    for (int j = 0; j < NOB; ++j) {
      double s = 0.0;
#pragma unroll
      for (int y = 0; y < ncart(LB); ++y) s = fma(c_trans[mode][LB][j][y], tmp[i][y], s);
      w[i][j] = s;
    }
}

// ---------------------------------------------------------------------------
// 3-centre (mu nu | P)
// ---------------------------------------------------------------------------

template <int LA, int LB, int LC, bool SPH>
__global__ void __launch_bounds__(Int3cCfg<LA, LB, LC, SPH>::THREADS, min_ctas3c(LA, LB, LC))
    int3c_kernel(DevBasis orb, DevBasis aux, const double* __restrict__ xyz,
                 const DevMol* __restrict__ mols, const int2* __restrict__ pairs,
                 const ClassMol* __restrict__ cms, int ncm, double* __restrict__ out) {
  using C = Int3cCfg<LA, LB, LC, SPH>;
  constexpr int NCA = ncart(LA), NCB = ncart(LB), NCC = ncart(LC);
  constexpr int NOA = C::NOA, NOB = C::NOB, NOC = C::NOC;
  constexpr int NR = (LA + LB + LC) / 2 + 1;
  constexpr int MODE = SPH ? 0 : 1;
  constexpr Cart<LA> ca{};
  constexpr Cart<LB> cb{};
  __shared__ double stage[C::SLOTS][NCC][NOA * NOB];

  const ClassMol cm = cms[find_cm(cms, ncm, blockIdx.x)];
  const int t0 = (blockIdx.x - cm.chunk_begin) * C::SLOTS;
  const int slot = threadIdx.x / NCC, kc = threadIdx.x % NCC;
  const int t = t0 + slot;
  const bool valid = t < cm.ntriples;

  double acc[NCA][NCB];
#pragma unroll
  for (int i = 0; i < NCA; ++i)
#pragma unroll
    for (int j = 0; j < NCB; ++j) acc[i][j] = 0.0;

  if (valid) {
    const int2 pr = pairs[cm.pair_begin + t / cm.naux];
    const int sc = cm.aux_begin + t % cm.naux;
    int kx, ky, kz;
    cart_of(LC, kc, kx, ky, kz);
    const double* A = xyz + 3 * orb.atom[pr.x];
    const double* B = xyz + 3 * orb.atom[pr.y];
    const double* Cc = xyz + 3 * aux.atom[sc];
    const double ab[3] = {A[0] - B[0], A[1] - B[1], A[2] - B[2]};
    const double rab2 = ab[0] * ab[0] + ab[1] * ab[1] + ab[2] * ab[2];
    const int pa0 = orb.prim_off[pr.x], na = orb.nprim[pr.x];
    const int pb0 = orb.prim_off[pr.y], nb = orb.nprim[pr.y];
    const int pc0 = aux.prim_off[sc], nc = aux.nprim[sc];
    for (int ia = 0; ia < na; ++ia) {
      const double a = orb.exps[pa0 + ia], ca_ = orb.coefs[pa0 + ia];
      for (int ib = 0; ib < nb; ++ib) {
        const double b = orb.exps[pb0 + ib], cb_ = orb.coefs[pb0 + ib];
        const double p = a + b, ip = 1.0 / p;
        const double kab = exp(-a * b * ip * rab2) * ca_ * cb_;
        if (fabs(kab) < kPrimPairCut) continue;
        const double P[3] = {(a * A[0] + b * B[0]) * ip, (a * A[1] + b * B[1]) * ip,
                             (a * A[2] + b * B[2]) * ip};
        for (int ic = 0; ic < nc; ++ic) {
          const double g = aux.exps[pc0 + ic], cg = aux.coefs[pc0 + ic];
          const double pq = p + g, ipq = 1.0 / pq;
          const double PQ[3] = {P[0] - Cc[0], P[1] - Cc[1], P[2] - Cc[2]};
          const double tt = p * g * ipq * (PQ[0] * PQ[0] + PQ[1] * PQ[1] + PQ[2] * PQ[2]);
          const double pref = 2.0 * kPi * kPi * sqrt(kPi) * ip / g * sqrt(ipq) * kab * cg;
          double u[NR], w[NR];
          rys_roots<NR>(tt, u, w);
#pragma unroll
          for (int r = 0; r < NR; ++r) {
            const double ur = u[r];
            const double qf = g * ipq * ur, pf = p * ipq * ur;
            const double b00 = 0.5 * ipq * ur;
            const double b10 = 0.5 * ip * (1.0 - qf);
            const double b01 = 0.5 / g * (1.0 - pf);
            double ix[LA + 1][LB + 1], iy[LA + 1][LB + 1], iz[LA + 1][LB + 1];
            rys_2d<LA, LB, LC>(P[0] - A[0] - qf * PQ[0], pf * PQ[0], b10, b01, b00, ab[0], kx, ix);
            rys_2d<LA, LB, LC>(P[1] - A[1] - qf * PQ[1], pf * PQ[1], b10, b01, b00, ab[1], ky, iy);
            rys_2d<LA, LB, LC>(P[2] - A[2] - qf * PQ[2], pf * PQ[2], b10, b01, b00, ab[2], kz, iz);
            const double wr = pref * w[r];
#pragma unroll
            for (int i = 0; i < NCA; ++i)
#pragma unroll
              for (int j = 0; j < NCB; ++j)
                acc[i][j] = fma(wr * ix[ca.x[i]][cb.x[j]],
                                iy[ca.y[i]][cb.y[j]] * iz[ca.z[i]][cb.z[j]], acc[i][j]);
          }
        }
      }
    }
  }
  double wsph[NOA][NOB];
  transform_ab<LA, LB, NOA, NOB>(MODE, acc, wsph);
  if (threadIdx.x < C::THREADS) {
#pragma unroll
    for (int i = 0; i < NOA; ++i)
#pragma unroll
      for (int j = 0; j < NOB; ++j) stage[slot][kc][i * NOB + j] = wsph[i][j];
  }
  __syncthreads();

  const DevMol mol = mols[cm.mol];
  constexpr int PER_IJ = C::SLOTS * NOC;
  constexpr int TOTAL = PER_IJ * NOA * NOB;
  for (int o = threadIdx.x; o < TOTAL; o += C::THREADS) {
    const int ij = o / PER_IJ, r = o - ij * PER_IJ;
    const int s = r / NOC, k = r - s * NOC;
    const int ts = t0 + s;
    if (ts >= cm.ntriples) continue;
    const int2 pr = pairs[cm.pair_begin + ts / cm.naux];
    const int sc = cm.aux_begin + ts % cm.naux;
    const int i = ij / NOB, j = ij - i * NOB;
    const int mu = orb.func_off[pr.x] + i, nu = orb.func_off[pr.y] + j;
    if (pr.x == pr.y && mu < nu) continue;
    double v = 0.0;
#pragma unroll
    for (int z = 0; z < NCC; ++z) v = fma(c_trans[MODE][LC][k][z], stage[s][z][ij], v);
    const long long hi = mu > nu ? mu : nu, lo = mu > nu ? nu : mu;
    const long long row = hi * (hi + 1) / 2 + lo;
    out[mol.a_off + row * mol.naux + aux.func_off[sc] + k] = v;
  }
}

// ---------------------------------------------------------------------------
// 3-centre (mu nu | P), root-parallel form for classes with few Cartesian
// products: one thread per (shell pair, aux shell, Rys root) instead of per
// Cartesian aux component.  The per-component kernel above evaluates the
// roots and the vertical tables once per component (NCC times the same
// work); here each thread evaluates only its own root and one vertical table
// per direction, then forms every aux component from it.  The roots' partial
// sums meet in shared memory; the epilogue is the component kernel's.  Same
// CTA work decomposition (SLOTS triples per CTA), so both forms share the
// plan's launch tables.
// ---------------------------------------------------------------------------

__host__ __device__ constexpr int nroots3c(int la, int lb, int lc) { return (la + lb + lc) / 2 + 1; }
// classes whose per-thread accumulators stay small and whose per-root
// partials fit the static shared-memory limit
__host__ __device__ constexpr bool use_root_parallel3c(int la, int lb, int lc, bool sph) {
  return lc >= 1 && ncart(la) * ncart(lb) * ncart(lc) <= 36 &&
         slots3c(la, lb, lc, sph) * nroots3c(la, lb, lc) * ncart(lc) * out_count(la, sph) *
                 out_count(lb, sph) * 8 <= 40 * 1024;
}
__host__ __device__ constexpr int rp_threads3c(int la, int lb, int lc, bool sph) {
  return (slots3c(la, lb, lc, sph) * nroots3c(la, lb, lc) + 31) / 32 * 32;
}

template <int LA, int LB, int LC, bool SPH>
__global__ void __launch_bounds__(rp_threads3c(LA, LB, LC, SPH), min_ctas_rp(rp_threads3c(LA, LB, LC, SPH)))
    int3c_rp_kernel(DevBasis orb, DevBasis aux, const double* __restrict__ xyz,
                    const DevMol* __restrict__ mols, const int2* __restrict__ pairs,
                    const ClassMol* __restrict__ cms, int ncm, double* __restrict__ out) {
  using C = Int3cCfg<LA, LB, LC, SPH>;
  constexpr int NCA = ncart(LA), NCB = ncart(LB), NCC = ncart(LC);
  constexpr int NOA = C::NOA, NOB = C::NOB, NOC = C::NOC;
  constexpr int NR = nroots3c(LA, LB, LC);
  constexpr int LAB = LA + LB;
  constexpr int MODE = SPH ? 0 : 1;
  constexpr Cart<LA> ca{};
  constexpr Cart<LB> cb{};
  constexpr Cart<LC> cc{};
  __shared__ double part[C::SLOTS][NR][NCC][NOA * NOB];

  const ClassMol cm = cms[find_cm(cms, ncm, blockIdx.x)];
  const int t0 = (blockIdx.x - cm.chunk_begin) * C::SLOTS;
  const int slot = threadIdx.x / NR, r = threadIdx.x % NR;
  const int t = t0 + slot;
  const bool valid = slot < C::SLOTS && t < cm.ntriples;

  double acc[NCC][NCA][NCB];
#pragma unroll
  for (int k = 0; k < NCC; ++k)
#pragma unroll
    for (int i = 0; i < NCA; ++i)
#pragma unroll
      for (int j = 0; j < NCB; ++j) acc[k][i][j] = 0.0;

  if (valid) {
    const int2 pr = pairs[cm.pair_begin + t / cm.naux];
    const int sc = cm.aux_begin + t % cm.naux;
    const double* A = xyz + 3 * orb.atom[pr.x];
    const double* B = xyz + 3 * orb.atom[pr.y];
    const double* Cc = xyz + 3 * aux.atom[sc];
    const double ab[3] = {A[0] - B[0], A[1] - B[1], A[2] - B[2]};
    const double rab2 = ab[0] * ab[0] + ab[1] * ab[1] + ab[2] * ab[2];
    const int pa0 = orb.prim_off[pr.x], na = orb.nprim[pr.x];
    const int pb0 = orb.prim_off[pr.y], nb = orb.nprim[pr.y];
    const int pc0 = aux.prim_off[sc], nc = aux.nprim[sc];
    for (int ia = 0; ia < na; ++ia) {
      const double a = orb.exps[pa0 + ia], ca_ = orb.coefs[pa0 + ia];
      for (int ib = 0; ib < nb; ++ib) {
        const double b = orb.exps[pb0 + ib], cb_ = orb.coefs[pb0 + ib];
        const double p = a + b, ip = 1.0 / p;
        const double kab = exp(-a * b * ip * rab2) * ca_ * cb_;
        if (fabs(kab) < kPrimPairCut) continue;
        const double P[3] = {(a * A[0] + b * B[0]) * ip, (a * A[1] + b * B[1]) * ip,
                             (a * A[2] + b * B[2]) * ip};
        for (int ic = 0; ic < nc; ++ic) {
          const double g = aux.exps[pc0 + ic], cg = aux.coefs[pc0 + ic];
          const double pq = p + g, ipq = 1.0 / pq;
          const double PQ[3] = {P[0] - Cc[0], P[1] - Cc[1], P[2] - Cc[2]};
          const double tt = p * g * ipq * (PQ[0] * PQ[0] + PQ[1] * PQ[1] + PQ[2] * PQ[2]);
          const double pref = 2.0 * kPi * kPi * sqrt(kPi) * ip / g * sqrt(ipq) * kab * cg;
          double ur, wr0;
          rys_root_one<NR>(tt, r, ur, wr0);
          const double qf = g * ipq * ur, pf = p * ipq * ur;
          const double b00 = 0.5 * ipq * ur;
          const double b10 = 0.5 * ip * (1.0 - qf);
          const double b01 = 0.5 / g * (1.0 - pf);
          double gx[LAB + 1][LC + 1], gy[LAB + 1][LC + 1], gz[LAB + 1][LC + 1];
          rys_vrr<LAB, LC>(P[0] - A[0] - qf * PQ[0], pf * PQ[0], b10, b01, b00, gx);
          rys_vrr<LAB, LC>(P[1] - A[1] - qf * PQ[1], pf * PQ[1], b10, b01, b00, gy);
          rys_vrr<LAB, LC>(P[2] - A[2] - qf * PQ[2], pf * PQ[2], b10, b01, b00, gz);
          const double wr = pref * wr0;
#pragma unroll
          for (int k = 0; k < NCC; ++k) {
            double ix[LA + 1][LB + 1], iy[LA + 1][LB + 1], iz[LA + 1][LB + 1];
            rys_hrr_col<LA, LB, LC>(gx, cc.x[k], ab[0], ix);
            rys_hrr_col<LA, LB, LC>(gy, cc.y[k], ab[1], iy);
            rys_hrr_col<LA, LB, LC>(gz, cc.z[k], ab[2], iz);
#pragma unroll
            for (int i = 0; i < NCA; ++i)
#pragma unroll
              for (int j = 0; j < NCB; ++j)
                acc[k][i][j] = fma(wr * ix[ca.x[i]][cb.x[j]], iy[ca.y[i]][cb.y[j]] * iz[ca.z[i]][cb.z[j]],
                                   acc[k][i][j]);
          }
        }
      }
    }
  }
  if (slot < C::SLOTS) {
#pragma unroll
    for (int k = 0; k < NCC; ++k) {
      double wsph[NOA][NOB];
      transform_ab<LA, LB, NOA, NOB>(MODE, acc[k], wsph);
#pragma unroll
      for (int i = 0; i < NOA; ++i)
#pragma unroll
        for (int j = 0; j < NOB; ++j) part[slot][r][k][i * NOB + j] = wsph[i][j];
    }
  }
  __syncthreads();

  const DevMol mol = mols[cm.mol];
  constexpr int PER_IJ = C::SLOTS * NOC;
  constexpr int TOTAL = PER_IJ * NOA * NOB;
  for (int o = threadIdx.x; o < TOTAL; o += blockDim.x) {
    const int ij = o / PER_IJ, rr = o - ij * PER_IJ;
    const int s = rr / NOC, k = rr - s * NOC;
    const int ts = t0 + s;
    if (ts >= cm.ntriples) continue;
    const int2 pr = pairs[cm.pair_begin + ts / cm.naux];
    const int sc = cm.aux_begin + ts % cm.naux;
    const int i = ij / NOB, j = ij - i * NOB;
    const int mu = orb.func_off[pr.x] + i, nu = orb.func_off[pr.y] + j;
    if (pr.x == pr.y && mu < nu) continue;
    double v = 0.0;
#pragma unroll
    for (int z = 0; z < NCC; ++z) {
      double sz = 0.0;
#pragma unroll
      for (int q = 0; q < NR; ++q) sz += part[s][q][z][ij];
      v = fma(c_trans[MODE][LC][k][z], sz, v);
    }
    const long long hi = mu > nu ? mu : nu, lo = mu > nu ? nu : mu;
    const long long row = hi * (hi + 1) / 2 + lo;
    out[mol.a_off + row * mol.naux + aux.func_off[sc] + k] = v;
  }
}

// ---------------------------------------------------------------------------
// 2-centre metric (P | Q): same machinery with a zero-exponent partner at P
// ---------------------------------------------------------------------------

template <int LA, int LC, bool SPH>
__global__ void __launch_bounds__(Int2cCfg<LA, LC, SPH>::THREADS)
    int2c_kernel(DevBasis aux, const double* __restrict__ xyz, const DevMol* __restrict__ mols,
                 const int2* __restrict__ pairs, const ClassMol* __restrict__ cms, int ncm,
                 double* __restrict__ out) {
  using C = Int2cCfg<LA, LC, SPH>;
  constexpr int NCA = ncart(LA), NCC = ncart(LC);
  constexpr int NOA = C::NOA, NOC = C::NOC;
  constexpr int NR = (LA + LC) / 2 + 1;
  constexpr int MODE = SPH ? 0 : 1;
  constexpr Cart<LA> ca{};
  __shared__ double stage[C::SLOTS][NCC][NOA];

  const ClassMol cm = cms[find_cm(cms, ncm, blockIdx.x)];
  const int t0 = (blockIdx.x - cm.chunk_begin) * C::SLOTS;
  const int slot = threadIdx.x / NCC, kc = threadIdx.x % NCC;
  const int t = t0 + slot;
  const bool valid = t < cm.ntriples;
  double acc[NCA][1];
#pragma unroll
  for (int i = 0; i < NCA; ++i) acc[i][0] = 0.0;
  if (valid) {
    const int2 pr = pairs[cm.pair_begin + t];
    int kx, ky, kz;
    cart_of(LC, kc, kx, ky, kz);
    const double* A = xyz + 3 * aux.atom[pr.x];
    const double* Cc = xyz + 3 * aux.atom[pr.y];
    const int pa0 = aux.prim_off[pr.x], na = aux.nprim[pr.x];
    const int pc0 = aux.prim_off[pr.y], nc = aux.nprim[pr.y];
    for (int ia = 0; ia < na; ++ia) {
      const double p = aux.exps[pa0 + ia], ca_ = aux.coefs[pa0 + ia];
      for (int ic = 0; ic < nc; ++ic) {
        const double g = aux.exps[pc0 + ic], cg = aux.coefs[pc0 + ic];
        const double pq = p + g, ipq = 1.0 / pq;
        const double PQ[3] = {A[0] - Cc[0], A[1] - Cc[1], A[2] - Cc[2]};
        const double tt = p * g * ipq * (PQ[0] * PQ[0] + PQ[1] * PQ[1] + PQ[2] * PQ[2]);
        const double pref = 2.0 * kPi * kPi * sqrt(kPi) / (p * g) * sqrt(ipq) * ca_ * cg;
        double u[NR], w[NR];
        rys_roots<NR>(tt, u, w);
#pragma unroll
        for (int r = 0; r < NR; ++r) {
          const double ur = u[r];
          const double qf = g * ipq * ur, pf = p * ipq * ur;
          const double b00 = 0.5 * ipq * ur, b10 = 0.5 / p * (1.0 - qf), b01 = 0.5 / g * (1.0 - pf);
          double ix[LA + 1][1], iy[LA + 1][1], iz[LA + 1][1];
          rys_2d<LA, 0, LC>(-qf * PQ[0], pf * PQ[0], b10, b01, b00, 0.0, kx, ix);
          rys_2d<LA, 0, LC>(-qf * PQ[1], pf * PQ[1], b10, b01, b00, 0.0, ky, iy);
          rys_2d<LA, 0, LC>(-qf * PQ[2], pf * PQ[2], b10, b01, b00, 0.0, kz, iz);
          const double wr = pref * w[r];
#pragma unroll
          for (int i = 0; i < NCA; ++i)
            acc[i][0] = fma(wr * ix[ca.x[i]][0], iy[ca.y[i]][0] * iz[ca.z[i]][0], acc[i][0]);
        }
      }
    }
  }
  double wsph[NOA][1];
  transform_ab<LA, 0, NOA, 1>(MODE, acc, wsph);
  if (threadIdx.x < C::THREADS) {
#pragma unroll
    for (int i = 0; i < NOA; ++i) stage[slot][kc][i] = wsph[i][0];
  }
  __syncthreads();
  const DevMol mol = mols[cm.mol];
  constexpr int TOTAL = C::SLOTS * NOC * NOA;
  for (int o = threadIdx.x; o < TOTAL; o += C::THREADS) {
    const int i = o / (C::SLOTS * NOC), r = o - i * (C::SLOTS * NOC);
    const int s = r / NOC, k = r - s * NOC;
    const int ts = t0 + s;
    if (ts >= cm.ntriples) continue;
    const int2 pr = pairs[cm.pair_begin + ts];
    if (pr.x == pr.y && i < k) continue;  // diagonal shell pair: each entry once
    double v = 0.0;
#pragma unroll
    for (int z = 0; z < NCC; ++z) v = fma(c_trans[MODE][LC][k][z], stage[s][z][i], v);
    const long long P = aux.func_off[pr.x] + i, Q = aux.func_off[pr.y] + k;
    out[mol.met_off + P * mol.naux + Q] = v;
    out[mol.met_off + Q * mol.naux + P] = v;
  }
}

// ---------------------------------------------------------------------------
// one-electron: overlap + kinetic (Obara-Saika 1-D), nuclear attraction (Rys)
// ---------------------------------------------------------------------------

template <int LA, int LB, int NOA, int NOB>
__device__ __forceinline__ void store_1e(int mode, const double (&acc)[ncart(LA)][ncart(LB)],
                                         const DevBasis& orb, int2 pr, const DevMol& mol,
                                         double* __restrict__ dst) {
  double wsph[NOA][NOB];
  transform_ab<LA, LB, NOA, NOB>(mode, acc, wsph);
  double* o = dst + mol.mat_off;
  const long long f0 = orb.func_off[pr.x], g0 = orb.func_off[pr.y];
#pragma unroll
  for (int i = 0; i < NOA; ++i)
#pragma unroll
    for (int j = 0; j < NOB; ++j) {
      const long long mu = f0 + i, nu = g0 + j;
      o[mu * mol.nao + nu] = wsph[i][j];
      o[nu * mol.nao + mu] = wsph[i][j];
    }
}

template <int LA, int LB, bool SPH>
__global__ void __launch_bounds__(128)
    int1e_kernel(DevBasis orb, const double* __restrict__ xyz, const double* __restrict__ charge,
                 const DevMol* __restrict__ mols, const int2* __restrict__ pairs,
                 const ClassMol* __restrict__ cms, int ncm, double* __restrict__ S,
                 double* __restrict__ T, double* __restrict__ V) {
  constexpr int NCA = ncart(LA), NCB = ncart(LB);
  constexpr int NOA = SPH ? nsph(LA) : NCA, NOB = SPH ? nsph(LB) : NCB;
  constexpr int NR = (LA + LB) / 2 + 1;
  constexpr int MODE = SPH ? 0 : 1;
  constexpr Cart<LA> ca{};
  constexpr Cart<LB> cb{};
  const ClassMol cm = cms[find_cm(cms, ncm, blockIdx.x)];
  const int t = (blockIdx.x - cm.chunk_begin) * 128 + threadIdx.x;
  if (t >= cm.ntriples) return;
  const DevMol mol = mols[cm.mol];
  const int2 pr = pairs[cm.pair_begin + t];
  const double* A = xyz + 3 * orb.atom[pr.x];
  const double* B = xyz + 3 * orb.atom[pr.y];
  const double ab[3] = {A[0] - B[0], A[1] - B[1], A[2] - B[2]};
  const double rab2 = ab[0] * ab[0] + ab[1] * ab[1] + ab[2] * ab[2];
  const int pa0 = orb.prim_off[pr.x], na = orb.nprim[pr.x];
  const int pb0 = orb.prim_off[pr.y], nb = orb.nprim[pr.y];
  double accs[NCA][NCB], acct[NCA][NCB], accv[NCA][NCB];
#pragma unroll
  for (int i = 0; i < NCA; ++i)
#pragma unroll
    for (int j = 0; j < NCB; ++j) accs[i][j] = acct[i][j] = accv[i][j] = 0.0;
  for (int ia = 0; ia < na; ++ia) {
    const double a = orb.exps[pa0 + ia], ca_ = orb.coefs[pa0 + ia];
    for (int ib = 0; ib < nb; ++ib) {
      const double b = orb.exps[pb0 + ib], cb_ = orb.coefs[pb0 + ib];
      const double p = a + b, ip = 1.0 / p;
      const double kab = exp(-a * b * ip * rab2) * ca_ * cb_;
      const double P[3] = {(a * A[0] + b * B[0]) * ip, (a * A[1] + b * B[1]) * ip,
                           (a * A[2] + b * B[2]) * ip};
      // overlap/kinetic 1-D tables
      double s1[3][LA + 1][LB + 3], t1[3][LA + 1][LB + 1];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const double xpa = P[d] - A[d], xpb = P[d] - B[d];
        double s[LA + 1][LB + 3];
        s[0][0] = sqrt(kPi * ip);
#pragma unroll
        for (int i = 0; i < LA; ++i)
          s[i + 1][0] = xpa * s[i][0] + (i > 0 ? i * 0.5 * ip * s[i > 0 ? i - 1 : 0][0] : 0.0);
#pragma unroll
        for (int j = 0; j < LB + 2; ++j)
#pragma unroll
          for (int i = 0; i <= LA; ++i) {
            double v = xpb * s[i][j];
            if (i > 0) v += i * 0.5 * ip * s[i > 0 ? i - 1 : 0][j];
            if (j > 0) v += j * 0.5 * ip * s[i][j > 0 ? j - 1 : 0];
            s[i][j + 1] = v;
          }
#pragma unroll
        for (int i = 0; i <= LA; ++i) {
#pragma unroll
          for (int j = 0; j < LB + 3; ++j) s1[d][i][j] = s[i][j];
#pragma unroll
          for (int j = 0; j <= LB; ++j) {
            double v = -2.0 * b * (2 * j + 1) * s[i][j] + 4.0 * b * b * s[i][j + 2];
            if (j >= 2) v += j * (j - 1) * s[i][j >= 2 ? j - 2 : 0];
            t1[d][i][j] = -0.5 * v;
          }
        }
      }
#pragma unroll
      for (int i = 0; i < NCA; ++i)
#pragma unroll
        for (int j = 0; j < NCB; ++j) {
          const double sx = s1[0][ca.x[i]][cb.x[j]], sy = s1[1][ca.y[i]][cb.y[j]],
                       sz = s1[2][ca.z[i]][cb.z[j]];
          accs[i][j] = fma(kab, sx * sy * sz, accs[i][j]);
          acct[i][j] = fma(kab,
                           t1[0][ca.x[i]][cb.x[j]] * sy * sz + sx * t1[1][ca.y[i]][cb.y[j]] * sz +
                               sx * sy * t1[2][ca.z[i]][cb.z[j]],
                           acct[i][j]);
        }
      // nuclear attraction, every nucleus of the molecule
      const double vpref = 2.0 * kPi * ip * kab;
      for (int c = 0; c < mol.natom; ++c) {
        const double* Cn = xyz + 3 * (mol.atom_off + c);
        const double zc = charge[mol.atom_off + c];
        const double PC[3] = {P[0] - Cn[0], P[1] - Cn[1], P[2] - Cn[2]};
        const double tt = p * (PC[0] * PC[0] + PC[1] * PC[1] + PC[2] * PC[2]);
        double u[NR], w[NR];
        rys_roots<NR>(tt, u, w);
#pragma unroll
        for (int r = 0; r < NR; ++r) {
          const double ur = u[r];
          const double b10 = 0.5 * ip * (1.0 - ur);
          double ix[LA + 1][LB + 1], iy[LA + 1][LB + 1], iz[LA + 1][LB + 1];
          rys_2d<LA, LB, 0>(P[0] - A[0] - ur * PC[0], 0.0, b10, 0.0, 0.0, ab[0], 0, ix);
          rys_2d<LA, LB, 0>(P[1] - A[1] - ur * PC[1], 0.0, b10, 0.0, 0.0, ab[1], 0, iy);
          rys_2d<LA, LB, 0>(P[2] - A[2] - ur * PC[2], 0.0, b10, 0.0, 0.0, ab[2], 0, iz);
          const double wr = -zc * vpref * w[r];
#pragma unroll
          for (int i = 0; i < NCA; ++i)
#pragma unroll
            for (int j = 0; j < NCB; ++j)
              accv[i][j] = fma(wr * ix[ca.x[i]][cb.x[j]],
                               iy[ca.y[i]][cb.y[j]] * iz[ca.z[i]][cb.z[j]], accv[i][j]);
        }
      }
    }
  }
  store_1e<LA, LB, NOA, NOB>(MODE, accs, orb, pr, mol, S);
  store_1e<LA, LB, NOA, NOB>(MODE, acct, orb, pr, mol, T);
  store_1e<LA, LB, NOA, NOB>(MODE, accv, orb, pr, mol, V);
}

// ---------------------------------------------------------------------------
// dispatch
// ---------------------------------------------------------------------------

template <int LA, int LB, int LC, bool SPH>
static void launch3(const ClassLaunch& cl, const KernelArgs& k, cudaStream_t st) {
  if constexpr (use_root_parallel3c(LA, LB, LC, SPH)) {
    int3c_rp_kernel<LA, LB, LC, SPH><<<cl.nblocks, rp_threads3c(LA, LB, LC, SPH), 0, st>>>(
        k.orb, k.aux, k.xyz, k.mols, cl.pairs, cl.cms, cl.ncm, k.out);
  } else {
    int3c_kernel<LA, LB, LC, SPH><<<cl.nblocks, Int3cCfg<LA, LB, LC, SPH>::THREADS, 0, st>>>(
        k.orb, k.aux, k.xyz, k.mols, cl.pairs, cl.cms, cl.ncm, k.out);
  }
}

template <int LA, int LC, bool SPH>
static void launch2(const ClassLaunch& cl, const KernelArgs& k, cudaStream_t st) {
  int2c_kernel<LA, LC, SPH><<<cl.nblocks, Int2cCfg<LA, LC, SPH>::THREADS, 0, st>>>(
      k.aux, k.xyz, k.mols, cl.pairs, cl.cms, cl.ncm, k.out);
}

template <int LA, int LB, bool SPH>
static void launch1(const ClassLaunch& cl, const KernelArgs& k, cudaStream_t st) {
  int1e_kernel<LA, LB, SPH><<<cl.nblocks, 128, 0, st>>>(k.orb, k.xyz, k.charge, k.mols, cl.pairs,
                                                        cl.cms, cl.ncm, k.out, k.out2, k.out3);
}

#define VQC_L3(LA, LB, LC)                                              \
  case (LA * 100 + LB * 10 + LC):                                       \
    if (sph) launch3<LA, LB, LC, true>(cl, k, st);                      \
    else launch3<LA, LB, LC, false>(cl, k, st);                         \
    return true;
#define VQC_L3C(LA, LB) VQC_L3(LA, LB, 0) VQC_L3(LA, LB, 1) VQC_L3(LA, LB, 2) VQC_L3(LA, LB, 3)

bool dispatch_int3c(const ClassLaunch& cl, const KernelArgs& k, bool sph, cudaStream_t st) {
  switch (cl.la * 100 + cl.lb * 10 + cl.lc) {
    VQC_L3C(0, 0) VQC_L3C(1, 0) VQC_L3C(1, 1) VQC_L3C(2, 0) VQC_L3C(2, 1) VQC_L3C(2, 2)
    VQC_L3C(3, 0) VQC_L3C(3, 1) VQC_L3C(3, 2) VQC_L3C(3, 3)
    default: return false;
  }
}

#define VQC_L2(LA, LC)                                                  \
  case (LA * 10 + LC):                                                  \
    if (sph) launch2<LA, LC, true>(cl, k, st);                          \
    else launch2<LA, LC, false>(cl, k, st);                             \
    return true;

bool dispatch_int2c(const ClassLaunch& cl, const KernelArgs& k, bool sph, cudaStream_t st) {
  switch (cl.la * 10 + cl.lc) {
    VQC_L2(0, 0) VQC_L2(1, 0) VQC_L2(1, 1) VQC_L2(2, 0) VQC_L2(2, 1) VQC_L2(2, 2)
    VQC_L2(3, 0) VQC_L2(3, 1) VQC_L2(3, 2) VQC_L2(3, 3)
    default: return false;
  }
}

#define VQC_L1(LA, LB)                                                  \
  case (LA * 10 + LB):                                                  \
    if (sph) launch1<LA, LB, true>(cl, k, st);                          \
    else launch1<LA, LB, false>(cl, k, st);                             \
    return true;

bool dispatch_int1e(const ClassLaunch& cl, const KernelArgs& k, bool sph, cudaStream_t st) {
  switch (cl.la * 10 + cl.lb) {
    VQC_L1(0, 0) VQC_L1(1, 0) VQC_L1(1, 1) VQC_L1(2, 0) VQC_L1(2, 1) VQC_L1(2, 2)
    VQC_L1(3, 0) VQC_L1(3, 1) VQC_L1(3, 2) VQC_L1(3, 3)
    default: return false;
  }
}

}  // namespace vqc
