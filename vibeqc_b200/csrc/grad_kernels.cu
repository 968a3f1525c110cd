// Derivative-contraction kernels of the DF-RHF gradient (FP64):
//   g += sum_{mu nu P} Abar[mu nu, P] d(mu nu|P)/dR     (3-centre)
//   g += sum_{P Q}    Mbar[P, Q]      d(P|Q)/dR          (2-centre)
//   g += sum_{mu nu}  D d(T+V) - W dS                     (one-electron)
// Derivatives of a Cartesian Gaussian about its centre use
// d/dA_x (x-A_x)^i e^{-a (x-A_x)^2} = 2a (x-A_x)^{i+1} - i (x-A_x)^{i-1}
// inside the primitive loop; the third centre follows from translational
// invariance (reference docs/developer/df_derivatives.md:44-49).
// Reference contractions: src/integrals/s_integrals.cpp:1073,1492 (DF),
// :2187 (one-electron); CUDA src/scf/cuda/df_shell_kernel.cuh:38 and
// the public adjoint generativeqc_system_df_gradient_cuda
// (src/api/c_api_df_gradient.cpp:11).
//
// Weights arrive in the output (spherical or Cartesian) basis; each thread
// maps its block to Cartesian components with the same transforms the value
// kernels use.  Per-atom sums are reduced across a warp (segmented by atom)
// before FP64 atomics.
#include "vqc_kernels.cuh"

namespace vqc {

namespace {

__device__ __forceinline__ void cart_of_g(int l, int k, int& x, int& y, int& z) {
  int rem = k, lx = l;
  while (rem > l - lx) {
    rem -= l - lx + 1;
    --lx;
  }
  x = lx;
  y = l - lx - rem;
  z = rem;
}

__device__ __forceinline__ int find_cm_g(const ClassMol* __restrict__ cms, int ncm, int block) {
  int lo = 0, hi = ncm - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (cms[mid].chunk_begin <= block) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Add v (3 components) to grad[3*key+d] across a full warp, segmented by runs
// of equal key in lane order; key < 0 contributes nothing.
__device__ __forceinline__ void warp_seg_add(double* __restrict__ grad, int key, double vx,
                                             double vy, double vz) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int prev = __shfl_up_sync(full, key, 1);
  const bool head = lane == 0 || prev != key;
  const unsigned heads = __ballot_sync(full, head);
  double v[3] = {vx, vy, vz};
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    double u0 = __shfl_up_sync(full, v[0], off);
    double u1 = __shfl_up_sync(full, v[1], off);
    double u2 = __shfl_up_sync(full, v[2], off);
    if (lane >= off) {
      // lanes (lane-off, lane] contain no head -> same segment
      const unsigned span = ((lane == 31) ? 0xffffffffu : ((2u << lane) - 1u)) &
                            ~((2u << (lane - off)) - 1u);
      if ((heads & span) == 0u) {
        v[0] += u0;
        v[1] += u1;
        v[2] += u2;
      }
    }
  }
  const int next = __shfl_down_sync(full, key, 1);
  const bool tail = lane == 31 || next != key;
  if (tail && key >= 0) {
    atomicAdd(grad + 3 * key + 0, v[0]);
    atomicAdd(grad + 3 * key + 1, v[1]);
    atomicAdd(grad + 3 * key + 2, v[2]);
  }
}

template <int LA, int LB, int NOA, int NOB>
__device__ __forceinline__ void weights_to_cart(int mode, const double (&w)[NOA][NOB],
                                                double (&c)[ncart(LA)][ncart(LB)]) {
  double tmp[ncart(LA)][NOB];
#pragma unroll
  for (int x = 0; x < ncart(LA); ++x)
#pragma unroll
    for (int j = 0; j < NOB; ++j) {
      double s = 0.0;
#pragma unroll
      for (int i = 0; i < NOA; ++i) s = fma(c_trans[mode][LA][i][x], w[i][j], s);
      tmp[x][j] = s;
    }
#pragma unroll
  for (int x = 0; x < ncart(LA); ++x)
#pragma unroll
    for (int y = 0; y < ncart(LB); ++y) {
      double s = 0.0;
#pragma unroll
      for (int j = 0; j < NOB; ++j) s = fma(c_trans[mode][LB][j][y], tmp[x][j], s);
      c[x][y] = s;
    }
}

}  // namespace

__host__ __device__ constexpr int round32(int n) { return (n + 31) / 32 * 32; }

// ---------------------------------------------------------------------------
// 3-centre derivative contraction
// ---------------------------------------------------------------------------

template <int LA, int LB, int LC, bool SPH>
__global__ void __launch_bounds__(round32(Int3cCfg<LA, LB, LC, SPH>::THREADS),
                                  min_ctas_grad3c(LA, LB, LC))
    grad3c_kernel(DevBasis orb, DevBasis aux, const double* __restrict__ xyz,
                  const DevMol* __restrict__ mols, const int2* __restrict__ pairs,
                  const ClassMol* __restrict__ cms, int ncm, const double* __restrict__ abar,
                  double* __restrict__ grad) {
  using C = Int3cCfg<LA, LB, LC, SPH>;
  constexpr int NCA = ncart(LA), NCB = ncart(LB), NCC = ncart(LC);
  constexpr int NOA = C::NOA, NOB = C::NOB, NOC = C::NOC;
  constexpr int NR = (LA + LB + LC + 1) / 2 + 1;
  constexpr int MODE = SPH ? 0 : 1;
  constexpr Cart<LA> ca{};
  constexpr Cart<LB> cb{};

  const ClassMol cm = cms[find_cm_g(cms, ncm, blockIdx.x)];
  const int t0 = (blockIdx.x - cm.chunk_begin) * C::SLOTS;
  const int slot = threadIdx.x / NCC, kc = threadIdx.x % NCC;
  const int t = t0 + slot;
  const bool valid = slot < C::SLOTS && t < cm.ntriples;
  double gA[3] = {0.0, 0.0, 0.0}, gB[3] = {0.0, 0.0, 0.0};
  int atomA = -1, atomB = -1, atomC = -1;
  if (valid) {
    const int2 pr = pairs[cm.pair_begin + t / cm.naux];
    const int sc = cm.aux_begin + t % cm.naux;
    atomA = orb.atom[pr.x];
    atomB = orb.atom[pr.y];
    atomC = aux.atom[sc];
    if (!(atomA == atomB && atomB == atomC)) {
      const DevMol mol = mols[cm.mol];
      int kx, ky, kz;
      cart_of_g(LC, kc, kx, ky, kz);
      // weights: Abar block for this Cartesian aux component, in Cartesian a, b
      double wsph[NOA][NOB];
      const int fa = orb.func_off[pr.x], fb = orb.func_off[pr.y], fc = aux.func_off[sc];
#pragma unroll
      for (int i = 0; i < NOA; ++i)
#pragma unroll
        for (int j = 0; j < NOB; ++j) {
          const long long mu = fa + i, nu = fb + j;
          const long long hi = mu > nu ? mu : nu, lo = mu > nu ? nu : mu;
          const double* row = abar + mol.a_off + (hi * (hi + 1) / 2 + lo) * mol.naux + fc;
          double s = 0.0;
#pragma unroll
          for (int k = 0; k < NOC; ++k) s = fma(c_trans[MODE][LC][k][kc], __ldg(row + k), s);
          wsph[i][j] = s;
        }
      double wc[NCA][NCB];
      weights_to_cart<LA, LB, NOA, NOB>(MODE, wsph, wc);
      const double pair_factor = (pr.x == pr.y) ? 1.0 : 2.0;
      const double* A = xyz + 3 * atomA;
      const double* B = xyz + 3 * atomB;
      const double* Cc = xyz + 3 * atomC;
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
            const double pref =
                2.0 * kPi * kPi * sqrt(kPi) * ip / g * sqrt(ipq) * kab * cg * pair_factor;
            double u[NR], w[NR];
            rys_roots<NR>(tt, u, w);
#pragma unroll
            for (int r = 0; r < NR; ++r) {
              const double ur = u[r];
              const double qf = g * ipq * ur, pf = p * ipq * ur;
              const double b00 = 0.5 * ipq * ur, b10 = 0.5 * ip * (1.0 - qf),
                           b01 = 0.5 / g * (1.0 - pf);
              double ix[LA + 2][LB + 2], iy[LA + 2][LB + 2], iz[LA + 2][LB + 2];
              rys_2d<LA + 1, LB + 1, LC>(P[0] - A[0] - qf * PQ[0], pf * PQ[0], b10, b01, b00, ab[0], kx, ix);
              rys_2d<LA + 1, LB + 1, LC>(P[1] - A[1] - qf * PQ[1], pf * PQ[1], b10, b01, b00, ab[1], ky, iy);
              rys_2d<LA + 1, LB + 1, LC>(P[2] - A[2] - qf * PQ[2], pf * PQ[2], b10, b01, b00, ab[2], kz, iz);
              const double wr = pref * w[r];
#pragma unroll
              for (int i = 0; i < NCA; ++i)
#pragma unroll
                for (int j = 0; j < NCB; ++j) {
                  const int ax = ca.x[i], ay = ca.y[i], az = ca.z[i];
                  const int bx = cb.x[j], by = cb.y[j], bz = cb.z[j];
                  const double x0 = ix[ax][bx], y0 = iy[ay][by], z0 = iz[az][bz];
                  const double dax = 2.0 * a * ix[ax + 1][bx] - (ax ? ax * ix[ax ? ax - 1 : 0][bx] : 0.0);
                  const double day = 2.0 * a * iy[ay + 1][by] - (ay ? ay * iy[ay ? ay - 1 : 0][by] : 0.0);
                  const double daz = 2.0 * a * iz[az + 1][bz] - (az ? az * iz[az ? az - 1 : 0][bz] : 0.0);
                  const double dbx = 2.0 * b * ix[ax][bx + 1] - (bx ? bx * ix[ax][bx ? bx - 1 : 0] : 0.0);
                  const double dby = 2.0 * b * iy[ay][by + 1] - (by ? by * iy[ay][by ? by - 1 : 0] : 0.0);
                  const double dbz = 2.0 * b * iz[az][bz + 1] - (bz ? bz * iz[az][bz ? bz - 1 : 0] : 0.0);
                  const double ww = wr * wc[i][j];
                  gA[0] = fma(ww, dax * y0 * z0, gA[0]);
                  gA[1] = fma(ww, x0 * day * z0, gA[1]);
                  gA[2] = fma(ww, x0 * y0 * daz, gA[2]);
                  gB[0] = fma(ww, dbx * y0 * z0, gB[0]);
                  gB[1] = fma(ww, x0 * dby * z0, gB[1]);
                  gB[2] = fma(ww, x0 * y0 * dbz, gB[2]);
                }
            }
          }
        }
      }
    }
  }
  warp_seg_add(grad, atomA, gA[0], gA[1], gA[2]);
  warp_seg_add(grad, atomB, gB[0], gB[1], gB[2]);
  warp_seg_add(grad, atomC, -(gA[0] + gB[0]), -(gA[1] + gB[1]), -(gA[2] + gB[2]));
}

// ---------------------------------------------------------------------------
// 3-centre derivative contraction, root-parallel form for classes with few
// Cartesian products: one thread per (shell pair, aux shell, Rys root) holds
// the weights of every aux component, evaluates its own root and one
// vertical table per direction, and contracts all components from it (the
// per-component kernel above repeats the roots and vertical tables for each
// component).  The roots of a slot are adjacent lanes with the same atoms,
// so the warp-segmented atomics sum them.  Same CTA work decomposition as the
// value kernels (the plan's launch tables are shared).
// ---------------------------------------------------------------------------

__host__ __device__ constexpr int nroots_g3c(int la, int lb, int lc) { return (la + lb + lc + 1) / 2 + 1; }
__host__ __device__ constexpr bool use_root_parallel_g3c(int la, int lb, int lc) {
  return lc >= 1 && ncart(la) * ncart(lb) * ncart(lc) <= 36;
}
__host__ __device__ constexpr int rp_threads_g3c(int la, int lb, int lc, bool sph) {
  return round32(slots3c(la, lb, lc, sph) * nroots_g3c(la, lb, lc));
}

template <int LA, int LB, int LC, bool SPH>
__global__ void __launch_bounds__(rp_threads_g3c(LA, LB, LC, SPH),
                                  min_ctas_rp(rp_threads_g3c(LA, LB, LC, SPH)))
    grad3c_rp_kernel(DevBasis orb, DevBasis aux, const double* __restrict__ xyz,
                     const DevMol* __restrict__ mols, const int2* __restrict__ pairs,
                     const ClassMol* __restrict__ cms, int ncm, const double* __restrict__ abar,
                     double* __restrict__ grad) {
  using C = Int3cCfg<LA, LB, LC, SPH>;
  constexpr int NCA = ncart(LA), NCB = ncart(LB), NCC = ncart(LC);
  constexpr int NOA = C::NOA, NOB = C::NOB, NOC = C::NOC;
  constexpr int NR = nroots_g3c(LA, LB, LC);
  constexpr int LAB1 = LA + LB + 2;  // vertical table height for the raised a and b
  constexpr int MODE = SPH ? 0 : 1;
  constexpr Cart<LA> ca{};
  constexpr Cart<LB> cb{};
  constexpr Cart<LC> cc{};

  const ClassMol cm = cms[find_cm_g(cms, ncm, blockIdx.x)];
  const int t0 = (blockIdx.x - cm.chunk_begin) * C::SLOTS;
  const int slot = threadIdx.x / NR, r = threadIdx.x % NR;
  const int t = t0 + slot;
  const bool valid = slot < C::SLOTS && t < cm.ntriples;
  // contraction weights of every Cartesian aux component, Cartesian in a and
  // b: one copy per slot in shared memory, formed by the slot's first root
  // thread and read by all of its roots (a register copy per root thread held
  // these kernels at 126-255 registers)
  __shared__ double wsh[C::SLOTS][NCC * NCA * NCB];
  double gA[3] = {0.0, 0.0, 0.0}, gB[3] = {0.0, 0.0, 0.0};
  int atomA = -1, atomB = -1, atomC = -1;
  int2 pr = make_int2(0, 0);
  int sc = 0;
  bool work = false;
  if (valid) {
    pr = pairs[cm.pair_begin + t / cm.naux];
    sc = cm.aux_begin + t % cm.naux;
    atomA = orb.atom[pr.x];
    atomB = orb.atom[pr.y];
    atomC = aux.atom[sc];
    work = !(atomA == atomB && atomB == atomC);
  }
  if (work && r == 0) {
    const DevMol mol = mols[cm.mol];
    const int fa = orb.func_off[pr.x], fb = orb.func_off[pr.y], fc = aux.func_off[sc];
    double wk[NOA][NOB][NOC];
#pragma unroll
    for (int i = 0; i < NOA; ++i)
#pragma unroll
      for (int j = 0; j < NOB; ++j) {
        const long long mu = fa + i, nu = fb + j;
        const long long hi = mu > nu ? mu : nu, lo = mu > nu ? nu : mu;
        const double* row = abar + mol.a_off + (hi * (hi + 1) / 2 + lo) * mol.naux + fc;
#pragma unroll
        for (int k = 0; k < NOC; ++k) wk[i][j][k] = __ldg(row + k);
      }
#pragma unroll
    for (int z = 0; z < NCC; ++z) {
      double wsph[NOA][NOB];
#pragma unroll
      for (int i = 0; i < NOA; ++i)
#pragma unroll
        for (int j = 0; j < NOB; ++j) {
          double s = 0.0;
#pragma unroll
          for (int k = 0; k < NOC; ++k) s = fma(c_trans[MODE][LC][k][z], wk[i][j][k], s);
          wsph[i][j] = s;
        }
      double wcz[NCA][NCB];
      weights_to_cart<LA, LB, NOA, NOB>(MODE, wsph, wcz);
#pragma unroll
      for (int i = 0; i < NCA; ++i)
#pragma unroll
        for (int j = 0; j < NCB; ++j) wsh[slot][(z * NCA + i) * NCB + j] = wcz[i][j];
    }
  }
  __syncthreads();
  if (work) {
    {
      const double pair_factor = (pr.x == pr.y) ? 1.0 : 2.0;
      const double* A = xyz + 3 * atomA;
      const double* B = xyz + 3 * atomB;
      const double* Cc = xyz + 3 * atomC;
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
            const double pref =
                2.0 * kPi * kPi * sqrt(kPi) * ip / g * sqrt(ipq) * kab * cg * pair_factor;
            double ur, wr0;
            rys_root_one<NR>(tt, r, ur, wr0);
            const double qf = g * ipq * ur, pf = p * ipq * ur;
            const double b00 = 0.5 * ipq * ur, b10 = 0.5 * ip * (1.0 - qf),
                         b01 = 0.5 / g * (1.0 - pf);
            double gx[LAB1 + 1][LC + 1], gy[LAB1 + 1][LC + 1], gz[LAB1 + 1][LC + 1];
            rys_vrr<LAB1, LC>(P[0] - A[0] - qf * PQ[0], pf * PQ[0], b10, b01, b00, gx);
            rys_vrr<LAB1, LC>(P[1] - A[1] - qf * PQ[1], pf * PQ[1], b10, b01, b00, gy);
            rys_vrr<LAB1, LC>(P[2] - A[2] - qf * PQ[2], pf * PQ[2], b10, b01, b00, gz);
            const double wr = pref * wr0;
#pragma unroll
            for (int z = 0; z < NCC; ++z) {
              double ix[LA + 2][LB + 2], iy[LA + 2][LB + 2], iz[LA + 2][LB + 2];
              rys_hrr_col<LA + 1, LB + 1, LC>(gx, cc.x[z], ab[0], ix);
              rys_hrr_col<LA + 1, LB + 1, LC>(gy, cc.y[z], ab[1], iy);
              rys_hrr_col<LA + 1, LB + 1, LC>(gz, cc.z[z], ab[2], iz);
#pragma unroll
              for (int i = 0; i < NCA; ++i)
#pragma unroll
                for (int j = 0; j < NCB; ++j) {
                  const int ax = ca.x[i], ay = ca.y[i], az = ca.z[i];
                  const int bx = cb.x[j], by = cb.y[j], bz = cb.z[j];
                  const double x0 = ix[ax][bx], y0 = iy[ay][by], z0 = iz[az][bz];
                  const double dax = 2.0 * a * ix[ax + 1][bx] - (ax ? ax * ix[ax ? ax - 1 : 0][bx] : 0.0);
                  const double day = 2.0 * a * iy[ay + 1][by] - (ay ? ay * iy[ay ? ay - 1 : 0][by] : 0.0);
                  const double daz = 2.0 * a * iz[az + 1][bz] - (az ? az * iz[az ? az - 1 : 0][bz] : 0.0);
                  const double dbx = 2.0 * b * ix[ax][bx + 1] - (bx ? bx * ix[ax][bx ? bx - 1 : 0] : 0.0);
                  const double dby = 2.0 * b * iy[ay][by + 1] - (by ? by * iy[ay][by ? by - 1 : 0] : 0.0);
                  const double dbz = 2.0 * b * iz[az][bz + 1] - (bz ? bz * iz[az][bz ? bz - 1 : 0] : 0.0);
                  const double ww = wr * wsh[slot][(z * NCA + i) * NCB + j];
                  gA[0] = fma(ww, dax * y0 * z0, gA[0]);
                  gA[1] = fma(ww, x0 * day * z0, gA[1]);
                  gA[2] = fma(ww, x0 * y0 * daz, gA[2]);
                  gB[0] = fma(ww, dbx * y0 * z0, gB[0]);
                  gB[1] = fma(ww, x0 * dby * z0, gB[1]);
                  gB[2] = fma(ww, x0 * y0 * dbz, gB[2]);
                }
            }
          }
        }
      }
    }
  }
  warp_seg_add(grad, atomA, gA[0], gA[1], gA[2]);
  warp_seg_add(grad, atomB, gB[0], gB[1], gB[2]);
  warp_seg_add(grad, atomC, -(gA[0] + gB[0]), -(gA[1] + gB[1]), -(gA[2] + gB[2]));
}

// ---------------------------------------------------------------------------
// 2-centre derivative contraction
// ---------------------------------------------------------------------------

template <int LA, int LC, bool SPH>
__global__ void __launch_bounds__(round32(Int2cCfg<LA, LC, SPH>::THREADS))
    grad2c_kernel(DevBasis aux, const double* __restrict__ xyz, const DevMol* __restrict__ mols,
                  const int2* __restrict__ pairs, const ClassMol* __restrict__ cms, int ncm,
                  const double* __restrict__ mbar, double* __restrict__ grad) {
  using C = Int2cCfg<LA, LC, SPH>;
  constexpr int NCA = ncart(LA), NCC = ncart(LC);
  constexpr int NOA = C::NOA, NOC = C::NOC;
  constexpr int NR = (LA + LC + 1) / 2 + 1;
  constexpr int MODE = SPH ? 0 : 1;
  constexpr Cart<LA> ca{};
  const ClassMol cm = cms[find_cm_g(cms, ncm, blockIdx.x)];
  const int t0 = (blockIdx.x - cm.chunk_begin) * C::SLOTS;
  const int slot = threadIdx.x / NCC, kc = threadIdx.x % NCC;
  const int t = t0 + slot;
  const bool valid = slot < C::SLOTS && t < cm.ntriples;
  double gA[3] = {0.0, 0.0, 0.0};
  int atomA = -1, atomC = -1;
  if (valid) {
    const int2 pr = pairs[cm.pair_begin + t];
    atomA = aux.atom[pr.x];
    atomC = aux.atom[pr.y];
    if (atomA != atomC) {
      const DevMol mol = mols[cm.mol];
      int kx, ky, kz;
      cart_of_g(LC, kc, kx, ky, kz);
      const int fa = aux.func_off[pr.x], fc = aux.func_off[pr.y];
      double wsph[NOA][1];
#pragma unroll
      for (int i = 0; i < NOA; ++i) {
        const double* row = mbar + mol.met_off + (long long)(fa + i) * mol.naux + fc;
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < NOC; ++k) s = fma(c_trans[MODE][LC][k][kc], __ldg(row + k), s);
        wsph[i][0] = s;
      }
      double wc[NCA][1];
      weights_to_cart<LA, 0, NOA, 1>(MODE, wsph, wc);
      const double* A = xyz + 3 * atomA;
      const double* Cc = xyz + 3 * atomC;
      const int pa0 = aux.prim_off[pr.x], na = aux.nprim[pr.x];
      const int pc0 = aux.prim_off[pr.y], nc = aux.nprim[pr.y];
      for (int ia = 0; ia < na; ++ia) {
        const double p = aux.exps[pa0 + ia], ca_ = aux.coefs[pa0 + ia];
        for (int ic = 0; ic < nc; ++ic) {
          const double g = aux.exps[pc0 + ic], cg = aux.coefs[pc0 + ic];
          const double pq = p + g, ipq = 1.0 / pq;
          const double PQ[3] = {A[0] - Cc[0], A[1] - Cc[1], A[2] - Cc[2]};
          const double tt = p * g * ipq * (PQ[0] * PQ[0] + PQ[1] * PQ[1] + PQ[2] * PQ[2]);
          const double pref = 4.0 * kPi * kPi * sqrt(kPi) / (p * g) * sqrt(ipq) * ca_ * cg;  // x2: (P|Q)+(Q|P)
          double u[NR], w[NR];
          rys_roots<NR>(tt, u, w);
#pragma unroll
          for (int r = 0; r < NR; ++r) {
            const double ur = u[r];
            const double qf = g * ipq * ur, pf = p * ipq * ur;
            const double b00 = 0.5 * ipq * ur, b10 = 0.5 / p * (1.0 - qf), b01 = 0.5 / g * (1.0 - pf);
            double ix[LA + 2][1], iy[LA + 2][1], iz[LA + 2][1];
            rys_2d<LA + 1, 0, LC>(-qf * PQ[0], pf * PQ[0], b10, b01, b00, 0.0, kx, ix);
            rys_2d<LA + 1, 0, LC>(-qf * PQ[1], pf * PQ[1], b10, b01, b00, 0.0, ky, iy);
            rys_2d<LA + 1, 0, LC>(-qf * PQ[2], pf * PQ[2], b10, b01, b00, 0.0, kz, iz);
            const double wr = pref * w[r];
#pragma unroll
            for (int i = 0; i < NCA; ++i) {
              const int ax = ca.x[i], ay = ca.y[i], az = ca.z[i];
              const double x0 = ix[ax][0], y0 = iy[ay][0], z0 = iz[az][0];
              const double dax = 2.0 * p * ix[ax + 1][0] - (ax ? ax * ix[ax ? ax - 1 : 0][0] : 0.0);
              const double day = 2.0 * p * iy[ay + 1][0] - (ay ? ay * iy[ay ? ay - 1 : 0][0] : 0.0);
              const double daz = 2.0 * p * iz[az + 1][0] - (az ? az * iz[az ? az - 1 : 0][0] : 0.0);
              const double ww = wr * wc[i][0];
              gA[0] = fma(ww, dax * y0 * z0, gA[0]);
              gA[1] = fma(ww, x0 * day * z0, gA[1]);
              gA[2] = fma(ww, x0 * y0 * daz, gA[2]);
            }
          }
        }
      }
      if (pr.x == pr.y) gA[0] = gA[1] = gA[2] = 0.0;  // unreachable: same atom
    }
  }
  warp_seg_add(grad, atomA, gA[0], gA[1], gA[2]);
  warp_seg_add(grad, atomC, -gA[0], -gA[1], -gA[2]);
}

// ---------------------------------------------------------------------------
// one-electron derivative contraction: D d(T + V) - W dS
// ---------------------------------------------------------------------------

template <int LA, int LB, bool SPH>
__global__ void __launch_bounds__(128)
    grad1e_kernel(DevBasis orb, const double* __restrict__ xyz, const double* __restrict__ charge,
                  const DevMol* __restrict__ mols, const int2* __restrict__ pairs,
                  const ClassMol* __restrict__ cms, int ncm, const double* __restrict__ dens,
                  const double* __restrict__ wdens, double* __restrict__ grad) {
  constexpr int NCA = ncart(LA), NCB = ncart(LB);
  constexpr int NOA = out_count(LA, SPH), NOB = out_count(LB, SPH);
  constexpr int NR = (LA + LB + 1) / 2 + 1;
  constexpr int MODE = SPH ? 0 : 1;
  constexpr Cart<LA> ca{};
  constexpr Cart<LB> cb{};
  const ClassMol cm = cms[find_cm_g(cms, ncm, blockIdx.x)];
  const int t = (blockIdx.x - cm.chunk_begin) * 128 + threadIdx.x;
  if (t >= cm.ntriples) return;
  const DevMol mol = mols[cm.mol];
  const int2 pr = pairs[cm.pair_begin + t];
  const int atomA = orb.atom[pr.x], atomB = orb.atom[pr.y];
  const double factor = (pr.x == pr.y) ? 1.0 : 2.0;
  double dw[NOA][NOB], ww[NOA][NOB];
  const long long fa = orb.func_off[pr.x], fb = orb.func_off[pr.y];
#pragma unroll
  for (int i = 0; i < NOA; ++i)
#pragma unroll
    for (int j = 0; j < NOB; ++j) {
      dw[i][j] = factor * __ldg(dens + mol.mat_off + (fa + i) * mol.nao + fb + j);
      ww[i][j] = factor * __ldg(wdens + mol.mat_off + (fa + i) * mol.nao + fb + j);
    }
  double dc[NCA][NCB], wc[NCA][NCB];
  weights_to_cart<LA, LB, NOA, NOB>(MODE, dw, dc);
  weights_to_cart<LA, LB, NOA, NOB>(MODE, ww, wc);
  const double* A = xyz + 3 * atomA;
  const double* B = xyz + 3 * atomB;
  const double ab[3] = {A[0] - B[0], A[1] - B[1], A[2] - B[2]};
  const double rab2 = ab[0] * ab[0] + ab[1] * ab[1] + ab[2] * ab[2];
  const int pa0 = orb.prim_off[pr.x], na = orb.nprim[pr.x];
  const int pb0 = orb.prim_off[pr.y], nb = orb.nprim[pr.y];
  double gst[3] = {0.0, 0.0, 0.0};  // d/dA of (D T - W S); B gets the negative
  double gvA[3] = {0.0, 0.0, 0.0}, gvB[3] = {0.0, 0.0, 0.0};
  for (int ia = 0; ia < na; ++ia) {
    const double a = orb.exps[pa0 + ia], ca_ = orb.coefs[pa0 + ia];
    for (int ib = 0; ib < nb; ++ib) {
      const double b = orb.exps[pb0 + ib], cb_ = orb.coefs[pb0 + ib];
      const double p = a + b, ip = 1.0 / p;
      const double kab = exp(-a * b * ip * rab2) * ca_ * cb_;
      const double P[3] = {(a * A[0] + b * B[0]) * ip, (a * A[1] + b * B[1]) * ip,
                           (a * A[2] + b * B[2]) * ip};
      if (atomA != atomB) {
        double s1[3][LA + 2][LB + 3], t1[3][LA + 2][LB + 1];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const double xpa = P[d] - A[d], xpb = P[d] - B[d];
          double s[LA + 2][LB + 3];
          s[0][0] = sqrt(kPi * ip);
#pragma unroll
          for (int i = 0; i < LA + 1; ++i)
            s[i + 1][0] = xpa * s[i][0] + (i > 0 ? i * 0.5 * ip * s[i > 0 ? i - 1 : 0][0] : 0.0);
#pragma unroll
          for (int j = 0; j < LB + 2; ++j)
#pragma unroll
            for (int i = 0; i <= LA + 1; ++i) {
              double v = xpb * s[i][j];
              if (i > 0) v += i * 0.5 * ip * s[i > 0 ? i - 1 : 0][j];
              if (j > 0) v += j * 0.5 * ip * s[i][j > 0 ? j - 1 : 0];
              s[i][j + 1] = v;
            }
#pragma unroll
          for (int i = 0; i <= LA + 1; ++i) {
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
            const int ax = ca.x[i], ay = ca.y[i], az = ca.z[i];
            const int bx = cb.x[j], by = cb.y[j], bz = cb.z[j];
            const double sx = s1[0][ax][bx], sy = s1[1][ay][by], sz = s1[2][az][bz];
            const double tx = t1[0][ax][bx], ty = t1[1][ay][by], tz = t1[2][az][bz];
            // derivative tables along each direction
            const double dsx = 2.0 * a * s1[0][ax + 1][bx] - (ax ? ax * s1[0][ax ? ax - 1 : 0][bx] : 0.0);
            const double dsy = 2.0 * a * s1[1][ay + 1][by] - (ay ? ay * s1[1][ay ? ay - 1 : 0][by] : 0.0);
            const double dsz = 2.0 * a * s1[2][az + 1][bz] - (az ? az * s1[2][az ? az - 1 : 0][bz] : 0.0);
            const double dtx = 2.0 * a * t1[0][ax + 1][bx] - (ax ? ax * t1[0][ax ? ax - 1 : 0][bx] : 0.0);
            const double dty = 2.0 * a * t1[1][ay + 1][by] - (ay ? ay * t1[1][ay ? ay - 1 : 0][by] : 0.0);
            const double dtz = 2.0 * a * t1[2][az + 1][bz] - (az ? az * t1[2][az ? az - 1 : 0][bz] : 0.0);
            const double wd = kab * dc[i][j], wo = kab * wc[i][j];
            // dS/dA_x = dsx sy sz ; dT/dA_x = dtx sy sz + dsx (ty sz + sy tz)
            gst[0] += wd * (dtx * sy * sz + dsx * (ty * sz + sy * tz)) - wo * dsx * sy * sz;
            gst[1] += wd * (dty * sx * sz + dsy * (tx * sz + sx * tz)) - wo * sx * dsy * sz;
            gst[2] += wd * (dtz * sx * sy + dsz * (tx * sy + sx * ty)) - wo * sx * sy * dsz;
          }
      }
      // nuclear attraction: basis-centre derivatives; the nucleus gets -(A+B)
      const double vpref = 2.0 * kPi * ip * kab;
      for (int c = 0; c < mol.natom; ++c) {
        const int atomC = mol.atom_off + c;
        const double* Cn = xyz + 3 * atomC;
        const double zc = charge[atomC];
        const double PC[3] = {P[0] - Cn[0], P[1] - Cn[1], P[2] - Cn[2]};
        const double tt = p * (PC[0] * PC[0] + PC[1] * PC[1] + PC[2] * PC[2]);
        double u[NR], w[NR];
        rys_roots<NR>(tt, u, w);
        double cA[3] = {0.0, 0.0, 0.0}, cB[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int r = 0; r < NR; ++r) {
          const double ur = u[r];
          const double b10 = 0.5 * ip * (1.0 - ur);
          double ix[LA + 2][LB + 2], iy[LA + 2][LB + 2], iz[LA + 2][LB + 2];
          rys_2d<LA + 1, LB + 1, 0>(P[0] - A[0] - ur * PC[0], 0.0, b10, 0.0, 0.0, ab[0], 0, ix);
          rys_2d<LA + 1, LB + 1, 0>(P[1] - A[1] - ur * PC[1], 0.0, b10, 0.0, 0.0, ab[1], 0, iy);
          rys_2d<LA + 1, LB + 1, 0>(P[2] - A[2] - ur * PC[2], 0.0, b10, 0.0, 0.0, ab[2], 0, iz);
          const double wr = -zc * vpref * w[r];
#pragma unroll
          for (int i = 0; i < NCA; ++i)
#pragma unroll
            for (int j = 0; j < NCB; ++j) {
              const int ax = ca.x[i], ay = ca.y[i], az = ca.z[i];
              const int bx = cb.x[j], by = cb.y[j], bz = cb.z[j];
              const double x0 = ix[ax][bx], y0 = iy[ay][by], z0 = iz[az][bz];
              const double dax = 2.0 * a * ix[ax + 1][bx] - (ax ? ax * ix[ax ? ax - 1 : 0][bx] : 0.0);
              const double day = 2.0 * a * iy[ay + 1][by] - (ay ? ay * iy[ay ? ay - 1 : 0][by] : 0.0);
              const double daz = 2.0 * a * iz[az + 1][bz] - (az ? az * iz[az ? az - 1 : 0][bz] : 0.0);
              const double dbx = 2.0 * b * ix[ax][bx + 1] - (bx ? bx * ix[ax][bx ? bx - 1 : 0] : 0.0);
              const double dby = 2.0 * b * iy[ay][by + 1] - (by ? by * iy[ay][by ? by - 1 : 0] : 0.0);
              const double dbz = 2.0 * b * iz[az][bz + 1] - (bz ? bz * iz[az][bz ? bz - 1 : 0] : 0.0);
              const double wd = wr * dc[i][j];
              cA[0] = fma(wd, dax * y0 * z0, cA[0]);
              cA[1] = fma(wd, x0 * day * z0, cA[1]);
              cA[2] = fma(wd, x0 * y0 * daz, cA[2]);
              cB[0] = fma(wd, dbx * y0 * z0, cB[0]);
              cB[1] = fma(wd, x0 * dby * z0, cB[1]);
              cB[2] = fma(wd, x0 * y0 * dbz, cB[2]);
            }
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          gvA[d] += cA[d];
          gvB[d] += cB[d];
          atomicAdd(grad + 3 * atomC + d, -(cA[d] + cB[d]));
        }
      }
    }
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    atomicAdd(grad + 3 * atomA + d, gst[d] + gvA[d]);
    atomicAdd(grad + 3 * atomB + d, -gst[d] + gvB[d]);
  }
}

// ---------------------------------------------------------------------------
// dispatch
// ---------------------------------------------------------------------------

template <int LA, int LB, int LC, bool SPH>
static void glaunch3(const ClassLaunch& cl, const KernelArgs& k, cudaStream_t st) {
  if constexpr (use_root_parallel_g3c(LA, LB, LC)) {
    grad3c_rp_kernel<LA, LB, LC, SPH><<<cl.nblocks, rp_threads_g3c(LA, LB, LC, SPH), 0, st>>>(
        k.orb, k.aux, k.xyz, k.mols, cl.pairs, cl.cms, cl.ncm, k.w1, k.grad);
  } else {
    grad3c_kernel<LA, LB, LC, SPH><<<cl.nblocks, round32(Int3cCfg<LA, LB, LC, SPH>::THREADS), 0, st>>>(
        k.orb, k.aux, k.xyz, k.mols, cl.pairs, cl.cms, cl.ncm, k.w1, k.grad);
  }
}

template <int LA, int LC, bool SPH>
static void glaunch2(const ClassLaunch& cl, const KernelArgs& k, cudaStream_t st) {
  grad2c_kernel<LA, LC, SPH><<<cl.nblocks, round32(Int2cCfg<LA, LC, SPH>::THREADS), 0, st>>>(
      k.aux, k.xyz, k.mols, cl.pairs, cl.cms, cl.ncm, k.w1, k.grad);
}

template <int LA, int LB, bool SPH>
static void glaunch1(const ClassLaunch& cl, const KernelArgs& k, cudaStream_t st) {
  grad1e_kernel<LA, LB, SPH><<<cl.nblocks, 128, 0, st>>>(k.orb, k.xyz, k.charge, k.mols, cl.pairs,
                                                          cl.cms, cl.ncm, k.w1, k.w2, k.grad);
}

#define VQC_G3(LA, LB, LC)                                              \
  case (LA * 100 + LB * 10 + LC):                                       \
    if (sph) glaunch3<LA, LB, LC, true>(cl, k, st);                     \
    else glaunch3<LA, LB, LC, false>(cl, k, st);                        \
    return true;
#define VQC_G3C(LA, LB) VQC_G3(LA, LB, 0) VQC_G3(LA, LB, 1) VQC_G3(LA, LB, 2) VQC_G3(LA, LB, 3)

bool dispatch_grad3c(const ClassLaunch& cl, const KernelArgs& k, bool sph, cudaStream_t st) {
  switch (cl.la * 100 + cl.lb * 10 + cl.lc) {
    VQC_G3C(0, 0) VQC_G3C(1, 0) VQC_G3C(1, 1) VQC_G3C(2, 0) VQC_G3C(2, 1) VQC_G3C(2, 2)
    VQC_G3C(3, 0) VQC_G3C(3, 1) VQC_G3C(3, 2) VQC_G3C(3, 3)
    default: return false;
  }
}

#define VQC_G2(LA, LC)                                                  \
  case (LA * 10 + LC):                                                  \
    if (sph) glaunch2<LA, LC, true>(cl, k, st);                         \
    else glaunch2<LA, LC, false>(cl, k, st);                            \
    return true;

bool dispatch_grad2c(const ClassLaunch& cl, const KernelArgs& k, bool sph, cudaStream_t st) {
  switch (cl.la * 10 + cl.lc) {
    VQC_G2(0, 0) VQC_G2(1, 0) VQC_G2(1, 1) VQC_G2(2, 0) VQC_G2(2, 1) VQC_G2(2, 2)
    VQC_G2(3, 0) VQC_G2(3, 1) VQC_G2(3, 2) VQC_G2(3, 3)
    default: return false;
  }
}

#define VQC_G1(LA, LB)                                                  \
  case (LA * 10 + LB):                                                  \
    if (sph) glaunch1<LA, LB, true>(cl, k, st);                         \
    else glaunch1<LA, LB, false>(cl, k, st);                            \
    return true;

bool dispatch_grad1e(const ClassLaunch& cl, const KernelArgs& k, bool sph, cudaStream_t st) {
  switch (cl.la * 10 + cl.lb) {
    VQC_G1(0, 0) VQC_G1(1, 0) VQC_G1(1, 1) VQC_G1(2, 0) VQC_G1(2, 1) VQC_G1(2, 2)
    VQC_G1(3, 0) VQC_G1(3, 1) VQC_G1(3, 2) VQC_G1(3, 3)
    default: return false;
  }
}

}  // namespace vqc
