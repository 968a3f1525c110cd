/*
 * CPU oracle for the DF-RHF integrals and their derivative contractions.
 *
 * TEST INFRASTRUCTURE ONLY: tests, the smoke check and the CPU-baseline leg of
 * the benchmark call this library as the checker. No product code path links
 * or loads it.
 *
 * It restates, with McMurchie-Davidson Hermite expansions (a method independent
 * of the Rys quadrature the CUDA kernels use), the integrals the reference
 * builds on the CPU:
 *   - S, T, V one-electron matrices       src/integrals/s_integrals.cpp:1865
 *   - 2-centre metric (P|Q) and 3-centre (mu nu|P) in the reference's layout
 *     A[(mu*N+nu)*X+P]                    src/integrals/s_integrals.cpp:1201
 *     followed by the real-spherical transform
 *                                         src/integrals/s_integrals.cpp:1520
 *   - the weighted DF derivative contraction
 *       g += sum Abar * d(mu nu|P) + sum Mbar * d(P|Q)
 *                                         src/integrals/s_integrals.cpp:1073,1492
 *   - the weighted one-electron derivative contraction
 *       g += sum D * dH - sum W * dS      src/integrals/s_integrals.cpp:2187
 * The third centre of every derivative follows from translational invariance,
 * as in docs/developer/df_derivatives.md:44-49 of the reference.
 *
 * Boys function: series F_m(T) = exp(-T) sum_k (2T)^k / ((2m+1)(2m+3)...(2m+2k+1))
 * with downward recursion for T < 30, F_0 from erf and upward recursion above.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define LMAX 6            /* per-centre angular momentum, raised included */
#define LTOT 16           /* total angular momentum in one R_tuv table */
#define NCMAX 28          /* ncart(LMAX) */
#define NSMAX 13          /* 2*LMAX+1 */

typedef struct {
  int nshell;
  const int *l, *atom, *nprim, *prim_off, *func_off;
  const double *exps, *coefs; /* coefficients with primitive+contraction norms */
  int nfunc;
  const double *trans;        /* [l][NSMAX][NCMAX] cart->output transform */
  const int *nout;            /* output functions per l (2l+1 or ncart) */
} oracle_basis;

static const double PI = 3.14159265358979323846;

static int ncart(int l) { return (l + 1) * (l + 2) / 2; }

static void cart_list(int l, int (*c)[3]) {
  int k = 0;
  for (int lx = l; lx >= 0; --lx)
    for (int ly = l - lx; ly >= 0; --ly) {
      c[k][0] = lx; c[k][1] = ly; c[k][2] = l - lx - ly; ++k;
    }
}

/* ---------------------------------------------------------------- Boys */
void oracle_boys(int mmax, double t, double *f) {
  if (t < 1e-14) {
    for (int m = 0; m <= mmax; ++m) f[m] = 1.0 / (2 * m + 1) - t / (2 * m + 3);
    return;
  }
  double et = exp(-t);
  if (t < 30.0) {
    double term = 1.0 / (2 * mmax + 1), sum = term;
    for (int k = 1; k < 400; ++k) {
      term *= 2.0 * t / (2 * mmax + 2 * k + 1);
      sum += term;
      if (term < 1e-18 * sum) break;
    }
    f[mmax] = et * sum;
    for (int m = mmax; m > 0; --m) f[m - 1] = (2.0 * t * f[m] + et) / (2 * m - 1);
  } else {
    f[0] = 0.5 * sqrt(PI / t) * erf(sqrt(t));
    for (int m = 0; m < mmax; ++m) f[m + 1] = ((2 * m + 1) * f[m] - et) / (2.0 * t);
  }
}

/* ------------------------------------------------ Hermite coefficients */
/* E[i][j][t] for one direction, i <= la, j <= lb, without exp prefactor. */
typedef double Etab[LMAX + 3][LMAX + 3][2 * LMAX + 7];

static void hermite_e(int la, int lb, double p, double xpa, double xpb, Etab e) {
  memset(e, 0, sizeof(Etab));
  double inv2p = 0.5 / p;
  e[0][0][0] = 1.0;
  for (int i = 0; i <= la; ++i) {
    for (int j = 0; j <= lb; ++j) {
      if (i == 0 && j == 0) continue;
      for (int t = 0; t <= i + j; ++t) {
        double v;
        if (j == 0) {
          v = xpa * e[i - 1][0][t] + (t + 1) * e[i - 1][0][t + 1];
          if (t > 0) v += inv2p * e[i - 1][0][t - 1];
        } else {
          v = xpb * e[i][j - 1][t] + (t + 1) * e[i][j - 1][t + 1];
          if (t > 0) v += inv2p * e[i][j - 1][t - 1];
        }
        e[i][j][t] = v;
      }
    }
  }
}

/* R_tuv(n=0) for t+u+v <= L; r[(t*(L+1)+u)*(L+1)+v]. work: (L+1)^4 doubles */
static void hermite_r(int L, double alpha, double x, double y, double z, double *r,
                      double *work) {
  int L1 = L + 1;
  double f[LTOT + 2];
  oracle_boys(L, alpha * (x * x + y * y + z * z), f);
#define RW(n, t, u, v) work[(((n) * L1 + (t)) * L1 + (u)) * L1 + (v)]
  double pw = 1.0;
  for (int n = 0; n <= L; ++n) {
    RW(n, 0, 0, 0) = pw * f[n];
    pw *= -2.0 * alpha;
  }
  for (int s = 1; s <= L; ++s) {
    for (int n = 0; n <= L - s; ++n) {
      for (int t = 0; t <= s; ++t)
        for (int u = 0; u <= s - t; ++u) {
          int v = s - t - u;
          double val;
          if (t > 0) {
            val = x * RW(n + 1, t - 1, u, v);
            if (t > 1) val += (t - 1) * RW(n + 1, t - 2, u, v);
          } else if (u > 0) {
            val = y * RW(n + 1, t, u - 1, v);
            if (u > 1) val += (u - 1) * RW(n + 1, t, u - 2, v);
          } else {
            val = z * RW(n + 1, t, u, v - 1);
            if (v > 1) val += (v - 1) * RW(n + 1, t, u, v - 2);
          }
          RW(n, t, u, v) = val;
        }
    }
  }
  for (int t = 0; t <= L; ++t)
    for (int u = 0; u <= L - t; ++u)
      for (int v = 0; v <= L - t - u; ++v) r[(t * L1 + u) * L1 + v] = RW(0, t, u, v);
#undef RW
}

/* ------------------------------------------- primitive 3-centre block */
/* out[(ia*ncart(lb)+ib)*ncart(lc)+ic] = (a b | c) for primitives; c alone. */
static void prim_eri3(int la, int lb, int lc, double a, const double *A, double b,
                      const double *B, double c, const double *C, double *out,
                      double *rbuf, double *work) {
  double p = a + b, mu = a * b / p;
  double P[3], ex[3][1];
  Etab E[3], Ec[3];
  double kab = 1.0;
  for (int d = 0; d < 3; ++d) {
    P[d] = (a * A[d] + b * B[d]) / p;
    double xab = A[d] - B[d];
    kab *= exp(-mu * xab * xab);
    hermite_e(la, lb, p, P[d] - A[d], P[d] - B[d], E[d]);
    hermite_e(lc, 0, c, 0.0, 0.0, Ec[d]);
    (void)ex;
  }
  double alpha = p * c / (p + c);
  int L = la + lb + lc, L1 = L + 1;
  hermite_r(L, alpha, P[0] - C[0], P[1] - C[1], P[2] - C[2], rbuf, work);
  double pref = 2.0 * pow(PI, 2.5) / (p * c * sqrt(p + c)) * kab;
  int ca[NCMAX][3], cb[NCMAX][3], cc[NCMAX][3];
  cart_list(la, ca); cart_list(lb, cb); cart_list(lc, cc);
  int na = ncart(la), nb = ncart(lb), nc = ncart(lc);
  int lab = la + lb, lab1 = lab + 1;
  double *w = work; /* reuse: W[t][u][v] for t,u,v <= lab */
  for (int ic = 0; ic < nc; ++ic) {
    int kx = cc[ic][0], ky = cc[ic][1], kz = cc[ic][2];
    for (int t = 0; t <= lab; ++t)
      for (int u = 0; u <= lab - t; ++u)
        for (int v = 0; v <= lab - t - u; ++v) {
          double s = 0.0;
          for (int tt = 0; tt <= kx; ++tt)
            for (int uu = 0; uu <= ky; ++uu)
              for (int vv = 0; vv <= kz; ++vv) {
                double ee = Ec[0][kx][0][tt] * Ec[1][ky][0][uu] * Ec[2][kz][0][vv];
                if (ee == 0.0) continue;
                double sg = ((tt + uu + vv) & 1) ? -1.0 : 1.0;
                s += sg * ee * rbuf[((t + tt) * L1 + (u + uu)) * L1 + (v + vv)];
              }
          w[(t * lab1 + u) * lab1 + v] = s;
        }
    for (int ia = 0; ia < na; ++ia)
      for (int ib = 0; ib < nb; ++ib) {
        double s = 0.0;
        int ax = ca[ia][0], ay = ca[ia][1], az = ca[ia][2];
        int bx = cb[ib][0], by = cb[ib][1], bz = cb[ib][2];
        for (int t = 0; t <= ax + bx; ++t) {
          double e1 = E[0][ax][bx][t];
          if (e1 == 0.0) continue;
          for (int u = 0; u <= ay + by; ++u) {
            double e2 = e1 * E[1][ay][by][u];
            if (e2 == 0.0) continue;
            for (int v = 0; v <= az + bz; ++v)
              s += e2 * E[2][az][bz][v] * w[(t * lab1 + u) * lab1 + v];
          }
        }
        out[(ia * nb + ib) * nc + ic] = pref * s;
      }
  }
}

/* ------------------------------------ primitive one-electron blocks */
/* overlap/kinetic 1D tables with extra j range for the kinetic operator */
static void prim_st(int la, int lb, double a, const double *A, double b, const double *B,
                    double *S, double *T) {
  double p = a + b, mu = a * b / p;
  Etab E[3];
  double s1[3][LMAX + 3][LMAX + 3], t1[3][LMAX + 3][LMAX + 3];
  for (int d = 0; d < 3; ++d) {
    double P = (a * A[d] + b * B[d]) / p, xab = A[d] - B[d];
    hermite_e(la, lb + 2, p, P - A[d], P - B[d], E[d]);
    double k = exp(-mu * xab * xab) * sqrt(PI / p);
    for (int i = 0; i <= la; ++i)
      for (int j = 0; j <= lb + 2; ++j) s1[d][i][j] = k * E[d][i][j][0];
    for (int i = 0; i <= la; ++i)
      for (int j = 0; j <= lb; ++j) {
        double v = -2.0 * b * (2 * j + 1) * s1[d][i][j] + 4.0 * b * b * s1[d][i][j + 2];
        if (j >= 2) v += j * (j - 1) * s1[d][i][j - 2];
        t1[d][i][j] = -0.5 * v;
      }
  }
  int ca[NCMAX][3], cb[NCMAX][3];
  cart_list(la, ca); cart_list(lb, cb);
  int na = ncart(la), nb = ncart(lb);
  for (int i = 0; i < na; ++i)
    for (int j = 0; j < nb; ++j) {
      double sx = s1[0][ca[i][0]][cb[j][0]], sy = s1[1][ca[i][1]][cb[j][1]],
             sz = s1[2][ca[i][2]][cb[j][2]];
      S[i * nb + j] = sx * sy * sz;
      if (T)
        T[i * nb + j] = t1[0][ca[i][0]][cb[j][0]] * sy * sz +
                        sx * t1[1][ca[i][1]][cb[j][1]] * sz +
                        sx * sy * t1[2][ca[i][2]][cb[j][2]];
    }
}

/* (a| 1/|r-C| |b) without the charge, for one nucleus */
static void prim_nuc(int la, int lb, double a, const double *A, double b, const double *B,
                     const double *C, double *V, double *rbuf, double *work) {
  double p = a + b, mu = a * b / p, P[3], kab = 1.0;
  Etab E[3];
  for (int d = 0; d < 3; ++d) {
    P[d] = (a * A[d] + b * B[d]) / p;
    double xab = A[d] - B[d];
    kab *= exp(-mu * xab * xab);
    hermite_e(la, lb, p, P[d] - A[d], P[d] - B[d], E[d]);
  }
  int L = la + lb, L1 = L + 1;
  hermite_r(L, p, P[0] - C[0], P[1] - C[1], P[2] - C[2], rbuf, work);
  double pref = 2.0 * PI / p * kab;
  int ca[NCMAX][3], cb[NCMAX][3];
  cart_list(la, ca); cart_list(lb, cb);
  int na = ncart(la), nb = ncart(lb);
  for (int i = 0; i < na; ++i)
    for (int j = 0; j < nb; ++j) {
      double s = 0.0;
      for (int t = 0; t <= ca[i][0] + cb[j][0]; ++t)
        for (int u = 0; u <= ca[i][1] + cb[j][1]; ++u)
          for (int v = 0; v <= ca[i][2] + cb[j][2]; ++v)
            s += E[0][ca[i][0]][cb[j][0]][t] * E[1][ca[i][1]][cb[j][1]][u] *
                 E[2][ca[i][2]][cb[j][2]][v] * rbuf[(t * L1 + u) * L1 + v];
      V[i * nb + j] = pref * s;
    }
}

/* --------------------------------------------------------- transforms */
static const double *tmat(const oracle_basis *bs, int l) {
  return bs->trans + (size_t)l * NSMAX * NCMAX;
}

/* out[i][j][k] (spherical) = Ta[i][x] Tb[j][y] Tc[k][z] in[x][y][z] */
static void transform3(const oracle_basis *ba, int la, const oracle_basis *bb, int lb,
                       const oracle_basis *bc, int lc, const double *in, double *out,
                       double *tmp) {
  int na = ncart(la), nb = ncart(lb), nc = ncart(lc);
  int oa = ba->nout[la], ob = bb->nout[lb], oc = bc->nout[lc];
  const double *Ta = tmat(ba, la), *Tb = tmat(bb, lb), *Tc = tmat(bc, lc);
  /* step 1: c */
  double *t1 = tmp, *t2 = tmp + na * nb * NSMAX;
  for (int x = 0; x < na * nb; ++x)
    for (int k = 0; k < oc; ++k) {
      double s = 0.0;
      for (int z = 0; z < nc; ++z) s += Tc[k * NCMAX + z] * in[x * nc + z];
      t1[x * oc + k] = s;
    }
  for (int x = 0; x < na; ++x)
    for (int j = 0; j < ob; ++j)
      for (int k = 0; k < oc; ++k) {
        double s = 0.0;
        for (int y = 0; y < nb; ++y) s += Tb[j * NCMAX + y] * t1[(x * nb + y) * oc + k];
        t2[(x * ob + j) * oc + k] = s;
      }
  for (int i = 0; i < oa; ++i)
    for (int j = 0; j < ob; ++j)
      for (int k = 0; k < oc; ++k) {
        double s = 0.0;
        for (int x = 0; x < na; ++x) s += Ta[i * NCMAX + x] * t2[(x * ob + j) * oc + k];
        out[(i * ob + j) * oc + k] = s;
      }
}

static void *xmalloc(size_t n) {
  void *p = malloc(n);
  if (!p) abort();
  return p;
}

#define WORK_DOUBLES ((LTOT + 1) * (LTOT + 1) * (LTOT + 1) * (LTOT + 1))

/* ------------------------------------------------------------ 3-centre */
/* Full (mu nu|P) tensor, out[(mu*N+nu)*X+P]. */
void oracle_int3c(const oracle_basis *orb, const oracle_basis *aux, const double *xyz,
                  double *out) {
  int N = orb->nfunc, X = aux->nfunc;
#pragma omp parallel
  {
    double *rbuf = xmalloc(sizeof(double) * WORK_DOUBLES);
    double *work = xmalloc(sizeof(double) * WORK_DOUBLES);
    double *prim = xmalloc(sizeof(double) * NCMAX * NCMAX * NCMAX);
    double *acc = xmalloc(sizeof(double) * NCMAX * NCMAX * NCMAX);
    double *sph = xmalloc(sizeof(double) * NCMAX * NCMAX * NCMAX);
    double *tmp = xmalloc(sizeof(double) * 2 * NCMAX * NCMAX * NCMAX);
#pragma omp for schedule(dynamic)
    for (int sa = 0; sa < orb->nshell; ++sa) {
      for (int sb = 0; sb <= sa; ++sb) {
        int la = orb->l[sa], lb = orb->l[sb];
        const double *A = xyz + 3 * orb->atom[sa], *B = xyz + 3 * orb->atom[sb];
        for (int sc = 0; sc < aux->nshell; ++sc) {
          int lc = aux->l[sc];
          const double *C = xyz + 3 * aux->atom[sc];
          int nblk = ncart(la) * ncart(lb) * ncart(lc);
          memset(acc, 0, sizeof(double) * nblk);
          for (int ia = 0; ia < orb->nprim[sa]; ++ia)
            for (int ib = 0; ib < orb->nprim[sb]; ++ib)
              for (int ic = 0; ic < aux->nprim[sc]; ++ic) {
                int pa = orb->prim_off[sa] + ia, pb = orb->prim_off[sb] + ib,
                    pc = aux->prim_off[sc] + ic;
                double cf = orb->coefs[pa] * orb->coefs[pb] * aux->coefs[pc];
                prim_eri3(la, lb, lc, orb->exps[pa], A, orb->exps[pb], B, aux->exps[pc], C,
                          prim, rbuf, work);
                for (int k = 0; k < nblk; ++k) acc[k] += cf * prim[k];
              }
          transform3(orb, la, orb, lb, aux, lc, acc, sph, tmp);
          int oa = orb->nout[la], ob = orb->nout[lb], oc = aux->nout[lc];
          int fa = orb->func_off[sa], fb = orb->func_off[sb], fc = aux->func_off[sc];
          for (int i = 0; i < oa; ++i)
            for (int j = 0; j < ob; ++j)
              for (int k = 0; k < oc; ++k) {
                double v = sph[(i * ob + j) * oc + k];
                out[((size_t)(fa + i) * N + (fb + j)) * X + fc + k] = v;
                out[((size_t)(fb + j) * N + (fa + i)) * X + fc + k] = v;
              }
        }
      }
    }
    free(rbuf); free(work); free(prim); free(acc); free(sph); free(tmp);
  }
}

/* ------------------------------------------------------------ 2-centre */
void oracle_int2c(const oracle_basis *aux, const double *xyz, double *out) {
  int X = aux->nfunc;
#pragma omp parallel
  {
    double *rbuf = xmalloc(sizeof(double) * WORK_DOUBLES);
    double *work = xmalloc(sizeof(double) * WORK_DOUBLES);
    double *prim = xmalloc(sizeof(double) * NCMAX * NCMAX);
    double *acc = xmalloc(sizeof(double) * NCMAX * NCMAX);
    double *sph = xmalloc(sizeof(double) * NCMAX * NCMAX);
    double *tmp = xmalloc(sizeof(double) * 2 * NCMAX * NCMAX * NSMAX);
    static const double one[1] = {1.0};
    (void)one;
#pragma omp for schedule(dynamic)
    for (int sa = 0; sa < aux->nshell; ++sa)
      for (int sb = 0; sb <= sa; ++sb) {
        int la = aux->l[sa], lb = aux->l[sb];
        const double *A = xyz + 3 * aux->atom[sa], *B = xyz + 3 * aux->atom[sb];
        int nblk = ncart(la) * ncart(lb);
        memset(acc, 0, sizeof(double) * nblk);
        for (int ia = 0; ia < aux->nprim[sa]; ++ia)
          for (int ib = 0; ib < aux->nprim[sb]; ++ib) {
            int pa = aux->prim_off[sa] + ia, pb = aux->prim_off[sb] + ib;
            /* (a|b) = (a s0|b) with a zero-exponent s partner at A */
            prim_eri3(la, 0, lb, aux->exps[pa], A, 0.0, A, aux->exps[pb], B, prim, rbuf,
                      work);
            double cf = aux->coefs[pa] * aux->coefs[pb];
            for (int k = 0; k < nblk; ++k) acc[k] += cf * prim[k];
          }
        /* reuse transform3 with a trivial middle index (l = 0, transform 1) */
        int oa = aux->nout[la], ob = aux->nout[lb];
        const double *Ta = tmat(aux, la), *Tb = tmat(aux, lb);
        int na = ncart(la), nb = ncart(lb);
        for (int i = 0; i < oa; ++i)
          for (int y = 0; y < nb; ++y) {
            double s = 0.0;
            for (int x = 0; x < na; ++x) s += Ta[i * NCMAX + x] * acc[x * nb + y];
            tmp[i * nb + y] = s;
          }
        for (int i = 0; i < oa; ++i)
          for (int j = 0; j < ob; ++j) {
            double s = 0.0;
            for (int y = 0; y < nb; ++y) s += Tb[j * NCMAX + y] * tmp[i * nb + y];
            sph[i * ob + j] = s;
          }
        int fa = aux->func_off[sa], fb = aux->func_off[sb];
        for (int i = 0; i < oa; ++i)
          for (int j = 0; j < ob; ++j) {
            out[(size_t)(fa + i) * X + fb + j] = sph[i * ob + j];
            out[(size_t)(fb + j) * X + fa + i] = sph[i * ob + j];
          }
      }
    free(rbuf); free(work); free(prim); free(acc); free(sph); free(tmp);
  }
}

/* 2-D transform helper: out[i][j] = Ta[i][x] Tb[j][y] in[x][y] */
static void transform2(const oracle_basis *ba, int la, const oracle_basis *bb, int lb,
                       const double *in, double *out, double *tmp) {
  int na = ncart(la), nb = ncart(lb), oa = ba->nout[la], ob = bb->nout[lb];
  const double *Ta = tmat(ba, la), *Tb = tmat(bb, lb);
  for (int i = 0; i < oa; ++i)
    for (int y = 0; y < nb; ++y) {
      double s = 0.0;
      for (int x = 0; x < na; ++x) s += Ta[i * NCMAX + x] * in[x * nb + y];
      tmp[i * nb + y] = s;
    }
  for (int i = 0; i < oa; ++i)
    for (int j = 0; j < ob; ++j) {
      double s = 0.0;
      for (int y = 0; y < nb; ++y) s += Tb[j * NCMAX + y] * tmp[i * nb + y];
      out[i * ob + j] = s;
    }
}

/* ------------------------------------------------------- one-electron */
void oracle_int1e(const oracle_basis *orb, int natom, const double *xyz,
                  const double *charges, double *S, double *T, double *V) {
  int N = orb->nfunc;
#pragma omp parallel
  {
    double *rbuf = xmalloc(sizeof(double) * WORK_DOUBLES);
    double *work = xmalloc(sizeof(double) * WORK_DOUBLES);
    double ps[NCMAX * NCMAX], pt[NCMAX * NCMAX], pv[NCMAX * NCMAX];
    double as[NCMAX * NCMAX], at[NCMAX * NCMAX], av[NCMAX * NCMAX];
    double os[NSMAX * NSMAX], tmp[NCMAX * NCMAX];
#pragma omp for schedule(dynamic)
    for (int sa = 0; sa < orb->nshell; ++sa)
      for (int sb = 0; sb <= sa; ++sb) {
        int la = orb->l[sa], lb = orb->l[sb];
        const double *A = xyz + 3 * orb->atom[sa], *B = xyz + 3 * orb->atom[sb];
        int nblk = ncart(la) * ncart(lb);
        memset(as, 0, sizeof(as)); memset(at, 0, sizeof(at)); memset(av, 0, sizeof(av));
        for (int ia = 0; ia < orb->nprim[sa]; ++ia)
          for (int ib = 0; ib < orb->nprim[sb]; ++ib) {
            int pa = orb->prim_off[sa] + ia, pb = orb->prim_off[sb] + ib;
            double a = orb->exps[pa], b = orb->exps[pb];
            double cf = orb->coefs[pa] * orb->coefs[pb];
            prim_st(la, lb, a, A, b, B, ps, pt);
            for (int k = 0; k < nblk; ++k) { as[k] += cf * ps[k]; at[k] += cf * pt[k]; }
            for (int c = 0; c < natom; ++c) {
              prim_nuc(la, lb, a, A, b, B, xyz + 3 * c, pv, rbuf, work);
              for (int k = 0; k < nblk; ++k) av[k] -= charges[c] * cf * pv[k];
            }
          }
        int oa = orb->nout[la], ob = orb->nout[lb];
        int fa = orb->func_off[sa], fb = orb->func_off[sb];
        double *arr[3] = {as, at, av};
        double *dst[3] = {S, T, V};
        for (int m = 0; m < 3; ++m) {
          transform2(orb, la, orb, lb, arr[m], os, tmp);
          for (int i = 0; i < oa; ++i)
            for (int j = 0; j < ob; ++j) {
              dst[m][(size_t)(fa + i) * N + fb + j] = os[i * ob + j];
              dst[m][(size_t)(fb + j) * N + fa + i] = os[i * ob + j];
            }
        }
      }
    free(rbuf); free(work);
  }
}

/* ------------------------------------------------ derivative helpers */
/* d/dA_x of a Cartesian block with index a first: block for la from raised
 * (la+1) and lowered (la-1) blocks. rest = product of the other dims. */
static void deriv_first(int la, double a, const double *up, const double *dn, int rest,
                        double *dx /* [3][ncart(la)*rest] */) {
  int ca[NCMAX][3], cu[NCMAX][3], cd[NCMAX][3];
  cart_list(la, ca); cart_list(la + 1, cu);
  if (la > 0) cart_list(la - 1, cd);
  int na = ncart(la), nu = ncart(la + 1), nd = la > 0 ? ncart(la - 1) : 0;
  for (int d = 0; d < 3; ++d)
    for (int i = 0; i < na; ++i) {
      int tu[3] = {ca[i][0], ca[i][1], ca[i][2]};
      tu[d] += 1;
      int iu = -1;
      for (int k = 0; k < nu; ++k)
        if (cu[k][0] == tu[0] && cu[k][1] == tu[1] && cu[k][2] == tu[2]) iu = k;
      int id = -1;
      if (ca[i][d] > 0) {
        int td[3] = {ca[i][0], ca[i][1], ca[i][2]};
        td[d] -= 1;
        for (int k = 0; k < nd; ++k)
          if (cd[k][0] == td[0] && cd[k][1] == td[1] && cd[k][2] == td[2]) id = k;
      }
      for (int r = 0; r < rest; ++r) {
        double v = 2.0 * a * up[iu * rest + r];
        if (id >= 0) v -= ca[i][d] * dn[id * rest + r];
        dx[(d * na + i) * rest + r] = v;
      }
    }
}

/* swap the first two indices of a [n1][n2][rest] block */
static void swap12(const double *in, int n1, int n2, int rest, double *out) {
  for (int i = 0; i < n1; ++i)
    for (int j = 0; j < n2; ++j)
      for (int r = 0; r < rest; ++r) out[(j * n1 + i) * rest + r] = in[(i * n2 + j) * rest + r];
}

/* --------------------------------------------- 3-centre gradient */
/* grad[3*natom] += sum_{mu nu P} abar[(mu*N+nu)*X+P] d(mu nu|P)/dR */
void oracle_grad3c(const oracle_basis *orb, const oracle_basis *aux, int natom,
                   const double *xyz, const double *abar, double *grad) {
  int N = orb->nfunc, X = aux->nfunc;
  int nthreads_max = 1;
#ifdef _OPENMP
  nthreads_max = omp_get_max_threads();
#endif
  double *gpriv = calloc((size_t)nthreads_max * 3 * natom, sizeof(double));
#pragma omp parallel
  {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    double *g = gpriv + (size_t)tid * 3 * natom;
    size_t big = (size_t)NCMAX * NCMAX * NCMAX;
    double *rbuf = xmalloc(sizeof(double) * WORK_DOUBLES);
    double *work = xmalloc(sizeof(double) * WORK_DOUBLES);
    double *up = xmalloc(sizeof(double) * big), *dn = xmalloc(sizeof(double) * big);
    double *t1 = xmalloc(sizeof(double) * big), *t2 = xmalloc(sizeof(double) * big);
    double *dA = xmalloc(sizeof(double) * 3 * big), *dB = xmalloc(sizeof(double) * 3 * big);
    double *dtmp = xmalloc(sizeof(double) * 3 * big);
    double *sph = xmalloc(sizeof(double) * big), *tmp = xmalloc(sizeof(double) * 2 * big);
#pragma omp for schedule(dynamic)
    for (int sa = 0; sa < orb->nshell; ++sa)
      for (int sb = 0; sb < orb->nshell; ++sb) {
        int la = orb->l[sa], lb = orb->l[sb];
        const double *A = xyz + 3 * orb->atom[sa], *B = xyz + 3 * orb->atom[sb];
        int na = ncart(la), nb = ncart(lb);
        for (int sc = 0; sc < aux->nshell; ++sc) {
          int lc = aux->l[sc], nc = ncart(lc);
          const double *C = xyz + 3 * aux->atom[sc];
          int blk = na * nb * nc;
          memset(dA, 0, sizeof(double) * 3 * blk);
          memset(dB, 0, sizeof(double) * 3 * blk);
          for (int ia = 0; ia < orb->nprim[sa]; ++ia)
            for (int ib = 0; ib < orb->nprim[sb]; ++ib)
              for (int ic = 0; ic < aux->nprim[sc]; ++ic) {
                int pa = orb->prim_off[sa] + ia, pb = orb->prim_off[sb] + ib,
                    pc = aux->prim_off[sc] + ic;
                double a = orb->exps[pa], b = orb->exps[pb], c = aux->exps[pc];
                double cf = orb->coefs[pa] * orb->coefs[pb] * aux->coefs[pc];
                /* centre A */
                prim_eri3(la + 1, lb, lc, a, A, b, B, c, C, up, rbuf, work);
                if (la > 0) prim_eri3(la - 1, lb, lc, a, A, b, B, c, C, dn, rbuf, work);
                deriv_first(la, a, up, dn, nb * nc, dtmp);
                for (int k = 0; k < 3 * blk; ++k) dA[k] += cf * dtmp[k];
                /* centre B: compute with b first, then swap */
                prim_eri3(lb + 1, la, lc, b, B, a, A, c, C, up, rbuf, work);
                if (lb > 0) prim_eri3(lb - 1, la, lc, b, B, a, A, c, C, dn, rbuf, work);
                deriv_first(lb, b, up, dn, na * nc, dtmp);
                for (int d = 0; d < 3; ++d) {
                  swap12(dtmp + (size_t)d * blk, nb, na, nc, t1);
                  for (int k = 0; k < blk; ++k) dB[d * blk + k] += cf * t1[k];
                }
              }
          int oa = orb->nout[la], ob = orb->nout[lb], oc = aux->nout[lc];
          int fa = orb->func_off[sa], fb = orb->func_off[sb], fc = aux->func_off[sc];
          for (int d = 0; d < 3; ++d) {
            double ga = 0.0, gb = 0.0;
            transform3(orb, la, orb, lb, aux, lc, dA + (size_t)d * blk, sph, tmp);
            for (int i = 0; i < oa; ++i)
              for (int j = 0; j < ob; ++j)
                for (int k = 0; k < oc; ++k)
                  ga += abar[((size_t)(fa + i) * N + fb + j) * X + fc + k] *
                        sph[(i * ob + j) * oc + k];
            transform3(orb, la, orb, lb, aux, lc, dB + (size_t)d * blk, sph, tmp);
            for (int i = 0; i < oa; ++i)
              for (int j = 0; j < ob; ++j)
                for (int k = 0; k < oc; ++k)
                  gb += abar[((size_t)(fa + i) * N + fb + j) * X + fc + k] *
                        sph[(i * ob + j) * oc + k];
            g[3 * orb->atom[sa] + d] += ga;
            g[3 * orb->atom[sb] + d] += gb;
            g[3 * aux->atom[sc] + d] -= ga + gb;
          }
          (void)t2;
        }
      }
    free(rbuf); free(work); free(up); free(dn); free(t1); free(t2); free(dA); free(dB);
    free(dtmp); free(sph); free(tmp);
  }
  for (int t = 0; t < nthreads_max; ++t)
    for (int k = 0; k < 3 * natom; ++k) grad[k] += gpriv[(size_t)t * 3 * natom + k];
  free(gpriv);
}

/* --------------------------------------------- 2-centre gradient */
void oracle_grad2c(const oracle_basis *aux, int natom, const double *xyz,
                   const double *mbar, double *grad) {
  int X = aux->nfunc;
  double *rbuf = xmalloc(sizeof(double) * WORK_DOUBLES);
  double *work = xmalloc(sizeof(double) * WORK_DOUBLES);
  double up[NCMAX * NCMAX * 2], dn[NCMAX * NCMAX * 2];
  double dA[3 * NCMAX * NCMAX], dt[3 * NCMAX * NCMAX], sph[NSMAX * NSMAX], tmp[NCMAX * NCMAX];
  for (int sa = 0; sa < aux->nshell; ++sa)
    for (int sb = 0; sb < aux->nshell; ++sb) {
      int la = aux->l[sa], lb = aux->l[sb], na = ncart(la), nb = ncart(lb);
      const double *A = xyz + 3 * aux->atom[sa], *B = xyz + 3 * aux->atom[sb];
      memset(dA, 0, sizeof(dA));
      for (int ia = 0; ia < aux->nprim[sa]; ++ia)
        for (int ib = 0; ib < aux->nprim[sb]; ++ib) {
          int pa = aux->prim_off[sa] + ia, pb = aux->prim_off[sb] + ib;
          double a = aux->exps[pa], b = aux->exps[pb], cf = aux->coefs[pa] * aux->coefs[pb];
          prim_eri3(la + 1, 0, lb, a, A, 0.0, A, b, B, up, rbuf, work);
          if (la > 0) prim_eri3(la - 1, 0, lb, a, A, 0.0, A, b, B, dn, rbuf, work);
          deriv_first(la, a, up, dn, nb, dt);
          for (int k = 0; k < 3 * na * nb; ++k) dA[k] += cf * dt[k];
        }
      int oa = aux->nout[la], ob = aux->nout[lb];
      int fa = aux->func_off[sa], fb = aux->func_off[sb];
      for (int d = 0; d < 3; ++d) {
        transform2(aux, la, aux, lb, dA + d * na * nb, sph, tmp);
        double ga = 0.0;
        for (int i = 0; i < oa; ++i)
          for (int j = 0; j < ob; ++j) ga += mbar[(size_t)(fa + i) * X + fb + j] * sph[i * ob + j];
        grad[3 * aux->atom[sa] + d] += ga;
        grad[3 * aux->atom[sb] + d] -= ga;
      }
    }
  free(rbuf); free(work);
}

/* --------------------------------------------- one-electron gradient */
/* grad += sum D * d(T+V) - sum W * dS, including the nuclear-position term */
void oracle_grad1e(const oracle_basis *orb, int natom, const double *xyz,
                   const double *charges, const double *dens, const double *wdens,
                   double *grad) {
  int N = orb->nfunc;
  double *rbuf = xmalloc(sizeof(double) * WORK_DOUBLES);
  double *work = xmalloc(sizeof(double) * WORK_DOUBLES);
  double su[NCMAX * NCMAX], sd[NCMAX * NCMAX], tu[NCMAX * NCMAX], td[NCMAX * NCMAX];
  double ds[3 * NCMAX * NCMAX], dtk[3 * NCMAX * NCMAX], tmp3[3 * NCMAX * NCMAX];
  double dva[3 * NCMAX * NCMAX], dvb[3 * NCMAX * NCMAX], tsw[NCMAX * NCMAX];
  double sph[NSMAX * NSMAX], tmp[NCMAX * NCMAX];
  for (int sa = 0; sa < orb->nshell; ++sa)
    for (int sb = 0; sb < orb->nshell; ++sb) {
      int la = orb->l[sa], lb = orb->l[sb], na = ncart(la), nb = ncart(lb);
      int blk = na * nb;
      const double *A = xyz + 3 * orb->atom[sa], *B = xyz + 3 * orb->atom[sb];
      int oa = orb->nout[la], ob = orb->nout[lb];
      int fa = orb->func_off[sa], fb = orb->func_off[sb];
      memset(ds, 0, sizeof(ds)); memset(dtk, 0, sizeof(dtk));
      for (int ia = 0; ia < orb->nprim[sa]; ++ia)
        for (int ib = 0; ib < orb->nprim[sb]; ++ib) {
          int pa = orb->prim_off[sa] + ia, pb = orb->prim_off[sb] + ib;
          double a = orb->exps[pa], b = orb->exps[pb], cf = orb->coefs[pa] * orb->coefs[pb];
          prim_st(la + 1, lb, a, A, b, B, su, tu);
          if (la > 0) prim_st(la - 1, lb, a, A, b, B, sd, td);
          deriv_first(la, a, su, sd, nb, tmp3);
          for (int k = 0; k < 3 * blk; ++k) ds[k] += cf * tmp3[k];
          deriv_first(la, a, tu, td, nb, tmp3);
          for (int k = 0; k < 3 * blk; ++k) dtk[k] += cf * tmp3[k];
        }
      for (int d = 0; d < 3; ++d) {
        double g = 0.0;
        transform2(orb, la, orb, lb, ds + d * blk, sph, tmp);
        for (int i = 0; i < oa; ++i)
          for (int j = 0; j < ob; ++j) g -= wdens[(size_t)(fa + i) * N + fb + j] * sph[i * ob + j];
        transform2(orb, la, orb, lb, dtk + d * blk, sph, tmp);
        for (int i = 0; i < oa; ++i)
          for (int j = 0; j < ob; ++j) g += dens[(size_t)(fa + i) * N + fb + j] * sph[i * ob + j];
        grad[3 * orb->atom[sa] + d] += g;
        grad[3 * orb->atom[sb] + d] -= g;
      }
      /* nuclear attraction: per nucleus C, centres A and B; C by invariance */
      for (int c = 0; c < natom; ++c) {
        const double *C = xyz + 3 * c;
        memset(dva, 0, sizeof(dva)); memset(dvb, 0, sizeof(dvb));
        for (int ia = 0; ia < orb->nprim[sa]; ++ia)
          for (int ib = 0; ib < orb->nprim[sb]; ++ib) {
            int pa = orb->prim_off[sa] + ia, pb = orb->prim_off[sb] + ib;
            double a = orb->exps[pa], b = orb->exps[pb];
            double cf = -charges[c] * orb->coefs[pa] * orb->coefs[pb];
            prim_nuc(la + 1, lb, a, A, b, B, C, su, rbuf, work);
            if (la > 0) prim_nuc(la - 1, lb, a, A, b, B, C, sd, rbuf, work);
            deriv_first(la, a, su, sd, nb, tmp3);
            for (int k = 0; k < 3 * blk; ++k) dva[k] += cf * tmp3[k];
            prim_nuc(lb + 1, la, b, B, a, A, C, su, rbuf, work);
            if (lb > 0) prim_nuc(lb - 1, la, b, B, a, A, C, sd, rbuf, work);
            deriv_first(lb, b, su, sd, na, tmp3);
            for (int d = 0; d < 3; ++d) {
              swap12(tmp3 + d * blk, nb, na, 1, tsw);
              for (int k = 0; k < blk; ++k) dvb[d * blk + k] += cf * tsw[k];
            }
          }
        for (int d = 0; d < 3; ++d) {
          double ga = 0.0, gb = 0.0;
          transform2(orb, la, orb, lb, dva + d * blk, sph, tmp);
          for (int i = 0; i < oa; ++i)
            for (int j = 0; j < ob; ++j) ga += dens[(size_t)(fa + i) * N + fb + j] * sph[i * ob + j];
          transform2(orb, la, orb, lb, dvb + d * blk, sph, tmp);
          for (int i = 0; i < oa; ++i)
            for (int j = 0; j < ob; ++j) gb += dens[(size_t)(fa + i) * N + fb + j] * sph[i * ob + j];
          grad[3 * orb->atom[sa] + d] += ga;
          grad[3 * orb->atom[sb] + d] += gb;
          grad[3 * c + d] -= ga + gb;
        }
      }
    }
  free(rbuf); free(work);
}
