// FP64-accurate products on the int8 tensor cores (Ozaki-style slicing).
//
// A product C = A B^T of FP64 matrices is formed from exact integer pieces:
// every row x of A (and of B) is scaled by a power of two 2^-e so that
// max |x| 2^-e < 1 and cut into `ns` signed 7-bit slices by repeated
// round-to-nearest,
//     x 2^-e = sum_{s=1..ns} a_s 2^-7s + r,   a_s in [-127, 127],  |r| <= 2^-7ns,
// (each step multiplies by 2^7, rounds, clamps and subtracts: all exact in
// FP64).  Then
//     (A B^T)[m][n] = 2^(ea[m] + eb[n]) sum_{g=2..ns+1} 2^-7g sum_{s+t=g} (a_s b_t^T)[m][n]
// up to the dropped terms s + t > ns + 1 and the remainders, ~2^-7ns of the
// row/column scales.  The integer products run on tcgen05.mma kind::i8 with
// exact int32 accumulation in TMEM (an accumulator sums at most ns slice pairs:
// K * ns * 127^2 < 2^31, K up to ~19,000 at ns = 7), one accumulator per g; only the final int32 -> FP64 scaling and
// the sum over g round.  Ozaki, Ogita, Oishi & Rump, Numer. Algorithms 59
// (2012) 95-118, describe the error-free splitting; this is its integer form.
//
// Used for the whitening of the 3-centre tensor, B = A W (reference
// src/scf/density_fitting.cpp:711-764, src/scf/cuda/df_plan_setup.cpp:34,70:
// there a cuBLAS FP64 GEMM), with the slice count chosen for the path's
// accuracy.
//
//   ozaki_gemm_kernel: one 128 x 64 output tile per CTA (the ns accumulators
//   take 448 of the 512 TMEM columns, so one CTA per SM).  Per 128-byte
//   K-block: warp 6 loads the ns B-slice tiles as one group (two groups in
//   flight), warp 0 loads the ns A-slice tiles one by one (six in flight) in
//   the interleaved order 0, ns-1, 1, ns-2, ... so that heavy (many pairs) and
//   light slices alternate; warp 1 issues the MMAs (A slice s with the B
//   slices t, s + t <= ns + 1, into accumulator g = s + t); warps 2-5 drain
//   the accumulators (TMEM -> int32 -> FP64), scale, stage the tile in the
//   idle A ring and store whole rows.
//   With `upper`, B[n][k] = 0 for k > n and a column tile reads only the
//   K-blocks below its last column.
#include <algorithm>

#include "tc_common.cuh"
#include "vqc_df.h"
#include "vqc_plan.hpp"

namespace vqc {
namespace oz {

using namespace vqc::tc;

constexpr int BM = 128;
constexpr int BN = 64;
constexpr int BKB = 128;  // K-block: 128 int8 = one 128-byte swizzle row = 4 MMA K-steps
constexpr int kMaxSlices = 7;
static_assert(BKB == 4 * 32, "the MMA issue loop is unrolled for four 32-byte K-steps per K-block");
constexpr int kARing = 6;
constexpr int kWRing = 2;
constexpr int A_TILE = BM * BKB;              // 16 KB
constexpr int B_TILE = BN * BKB;              // 8 KB
constexpr int B_GROUP = kMaxSlices * B_TILE;  // 56 KB
// MMA issuers: the int8 MMA costs ~150 cycles of issue per instruction whatever its N, so
// two issuing warps (accumulators split by parity) keep more of them in flight
constexpr int kIssuers = 2;
constexpr int kThreads = 32 * (7 + kIssuers - 1);  // A producer, issuer 0, 4 epilogue, B producer, issuer 1
constexpr int kTmemCols = 512;                // ns (<= 7) accumulators of BN columns

struct OzCtrl {
  uint64_t a_full[kARing], a_empty[kARing], b_full[kWRing], b_empty[kWRing], acc_full, tmem_empty,
      drain;
  uint32_t tmem;
  int abort;
  int a_issued, a_consumed, b_issued, b_consumed;
};

constexpr int SMEM = kARing * A_TILE + kWRing * B_GROUP + 1024 + (int)sizeof(OzCtrl) + 64;
static_assert(SMEM <= 227 * 1024, "shared memory per CTA");

struct OzParams {
  int m, n, k, ns, upper, ntn, ntm, ntiles;
  int sym;       // symmetric output (A == B, m == n): only tiles reaching the diagonal or above
  int sym_per;   // tiles per molecule in the symmetric layout
  const int* a_exp;  // [nmol][m]
  const int* b_exp;  // [nmol][n]
  double* c;
  long long ldc, c_mol_stride;
  int* error;
};

// tile t -> (molecule, row tile, column tile), column tile fastest (CTAs that
// run together share an A row block in L2)
__device__ __forceinline__ void tile_coords(const OzParams& p, int t, int& z, int& tm, int& tn) {
  if (p.sym) {
    // row tile tm holds column tiles 2 tm .. ntn - 1 (BM = 2 BN): the tiles
    // that reach the diagonal or lie above it
    z = t / p.sym_per;
    int r = t - z * p.sym_per;
    tm = 0;
    while (r >= p.ntn - 2 * tm) {
      r -= p.ntn - 2 * tm;
      ++tm;
    }
    tn = 2 * tm + r;
    return;
  }
  tn = t % p.ntn;
  const int r = t / p.ntn;
  tm = r % p.ntm;
  z = r / p.ntm;
}
static_assert(BM == 2 * BN, "the symmetric tile layout pairs one row tile with two column tiles");

__device__ __forceinline__ int tile_kblocks(const OzParams& p, int tn) {
  const int kend = p.upper ? min(p.k, tn * BN + BN) : p.k;
  return (kend + BKB - 1) / BKB;
}

__device__ __forceinline__ void oz_abort(OzCtrl* c, int* error, int code) {
  if (error) atomicExch(error, code);
  *reinterpret_cast<volatile int*>(&c->abort) = 1;
}

__device__ __forceinline__ bool oz_aborted(OzCtrl* c) {
  return *reinterpret_cast<volatile int*>(&c->abort) != 0;
}

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                       uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// accumulate into D (no predicate to set up)
__device__ __forceinline__ void mma_i8_acc(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                           uint32_t idesc) {
  asm volatile("tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, 1;" ::"r"(tmem_d), "l"(adesc),
               "l"(bdesc), "r"(idesc)
               : "memory");
}

// 32 consecutive columns of a lane quarter, without waiting (tcgen05.wait::ld
// follows once all loads of an accumulator are in flight)
__device__ __forceinline__ void tmem_ld32_i32_nowait(uint32_t taddr, int* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, "
      "%30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]),
        "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]),
        "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = (int)r[i];
}

__device__ __forceinline__ void tmem_ld16_i32(uint32_t taddr, int (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = (int)r[i];
}

// j-th A slice of a K-block in issue order: 0, ns-1, 1, ns-2, ...
__device__ __forceinline__ int slice_order(int j, int ns) { return (j & 1) ? ns - 1 - (j >> 1) : (j >> 1); }

// D = S32 (bits 4-5 = 2), A = B = signed 8-bit (1), both K-major, N >> 3, M >> 4
constexpr uint32_t kIdescI8 = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                              ((uint32_t)(BM >> 4) << 24);


// Persistent over output tiles: each CTA (one per SM: 512 TMEM columns)
// takes tiles blockIdx.x, blockIdx.x + gridDim.x, ...  The producers run ahead
// across tile boundaries, so the next tile's operands are in flight while the
// epilogue drains the last one; the MMA issuer waits only until the epilogue
// has read TMEM (tmem_empty), and the epilogue's FP64 scaling and stores
// overlap the next tile's MMAs.
__global__ void __launch_bounds__(kThreads, 1)
    ozaki_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                      OzParams p) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  uint8_t* abuf = smem;
  uint8_t* bbuf = smem + kARing * A_TILE;
  OzCtrl* ctrl = reinterpret_cast<OzCtrl*>(bbuf + kWRing * B_GROUP);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int ns = p.ns;

  const uint32_t af0 = smem_u32(ctrl->a_full), ae0 = smem_u32(ctrl->a_empty);
  const uint32_t bf0 = smem_u32(ctrl->b_full), be0 = smem_u32(ctrl->b_empty);
  const uint32_t accf = smem_u32(&ctrl->acc_full), tmem_empty = smem_u32(&ctrl->tmem_empty);
  const uint32_t drain = smem_u32(&ctrl->drain);
  if (tid == 0) {
    for (int s = 0; s < kARing; ++s) {
      mbar_init(af0 + 8 * s, 1);
      mbar_init(ae0 + 8 * s, kIssuers);
    }
    for (int s = 0; s < kWRing; ++s) {
      mbar_init(bf0 + 8 * s, 1);
      mbar_init(be0 + 8 * s, kIssuers);
    }
    mbar_init(accf, kIssuers);
    mbar_init(tmem_empty, 4);  // one arrival per epilogue warp
    mbar_init(drain, kIssuers);
    ctrl->abort = 0;
    ctrl->a_issued = ctrl->a_consumed = ctrl->b_issued = ctrl->b_consumed = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&ctrl->tmem)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = ctrl->tmem;
  volatile int* ab = &ctrl->abort;

  if (warp == 6) {
    if (lane == 0) {  // B-slice groups, one per K-block of every tile
      int gkb = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < p.ntiles && ok && !oz_aborted(ctrl); t += gridDim.x) {
        int z, tm, tn;
        tile_coords(p, t, z, tm, tn);
        const int nkb = tile_kblocks(p, tn);
        for (int kb = 0; kb < nkb; ++kb, ++gkb) {
          const int ws = gkb % kWRing;
          if (gkb >= kWRing && !mbar_wait(be0 + 8 * ws, ((gkb / kWRing) - 1) & 1, ab)) {
            oz_abort(ctrl, p.error, 41);
            ok = false;
            break;
          }
          mbar_expect_tx(bf0 + 8 * ws, ns * B_TILE);
          for (int s = 0; s < ns; ++s)
            tma_load_3d(smem_u32(bbuf + ws * B_GROUP + s * B_TILE), &tmB, kb * BKB, tn * BN,
                        z * ns + s, bf0 + 8 * ws);
          *reinterpret_cast<volatile int*>(&ctrl->b_issued) = gkb + 1;
        }
      }
    }
  } else if (warp == 0) {
    if (lane == 0) {  // A-slice tiles in the interleaved slice order
      int ai = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < p.ntiles && ok && !oz_aborted(ctrl); t += gridDim.x) {
        int z, tm, tn;
        tile_coords(p, t, z, tm, tn);
        const int nkb = tile_kblocks(p, tn);
        for (int kb = 0; kb < nkb && ok; ++kb) {
          for (int j = 0; j < ns; ++j, ++ai) {
            const int as = ai % kARing;
            if (ai >= kARing && !mbar_wait(ae0 + 8 * as, ((ai / kARing) - 1) & 1, ab)) {
              oz_abort(ctrl, p.error, 42);
              ok = false;
              break;
            }
            mbar_expect_tx(af0 + 8 * as, A_TILE);
            tma_load_3d(smem_u32(abuf + as * A_TILE), &tmA, kb * BKB, tm * BM,
                        z * ns + slice_order(j, ns), af0 + 8 * as);
            *reinterpret_cast<volatile int*>(&ctrl->a_issued) = ai + 1;
          }
        }
      }
    }
  } else if (warp == 1 || warp >= 7) {
    const int me = warp == 1 ? 0 : warp - 6;  // issuer index: accumulators g with g % kIssuers == me
    if (lane == 0) {  // MMA issuer
      int ai = 0, gkb = 0, it = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < p.ntiles && ok && !oz_aborted(ctrl); t += gridDim.x, ++it) {
        int z, tm, tn;
        tile_coords(p, t, z, tm, tn);
        const int nkb = tile_kblocks(p, tn);
        // the epilogue has read the previous tile's accumulators
        if (it > 0 && !mbar_wait(tmem_empty, (it - 1) & 1, ab)) {
          oz_abort(ctrl, p.error, 46);
          break;
        }
        fence_after_sync();
        for (int kb = 0; kb < nkb && ok; ++kb, ++gkb) {
          const int ws = gkb % kWRing;
          if (!mbar_wait(bf0 + 8 * ws, (gkb / kWRing) & 1, ab)) {
            oz_abort(ctrl, p.error, 43);
            ok = false;
            break;
          }
          if (me == 0) *reinterpret_cast<volatile int*>(&ctrl->b_consumed) = gkb + 1;
          // descriptors advance by (byte offset >> 4) in their address field
          // (shared-memory addresses < 256 KB never carry out of it)
          const uint64_t bdesc0 = smem_desc(smem_u32(bbuf + ws * B_GROUP));
          for (int j = 0; j < ns; ++j, ++ai) {
            const int s = slice_order(j, ns);
            const int as = ai % kARing;
            if (!mbar_wait(af0 + 8 * as, (ai / kARing) & 1, ab)) {
              oz_abort(ctrl, p.error, 44);
              ok = false;
              break;
            }
            if (me == 0) *reinterpret_cast<volatile int*>(&ctrl->a_consumed) = ai + 1;
            fence_after_sync();
            // slices are 0-based here: pair (s, t) with s + t <= ns - 1 feeds
            // accumulator g = s + t (weight 2^-7(g+2)); slice 0 comes first in
            // the issue order, so its first K-step initialises every accumulator
            const uint64_t adesc0 = smem_desc(smem_u32(abuf + as * A_TILE));
            const uint32_t first = (kb == 0 && s == 0) ? 0u : 1u;
            uint32_t dt = tmem + (uint32_t)(s * BN);
            uint64_t bdesc = bdesc0;
            for (int tt = 0; tt + s < ns; ++tt, dt += BN, bdesc += B_TILE >> 4) {
              if ((s + tt) % kIssuers != me) continue;
              if (first) mma_i8_acc(dt, adesc0, bdesc, kIdescI8);
              else mma_i8(dt, adesc0, bdesc, kIdescI8, 0u);
              mma_i8_acc(dt, adesc0 + 2, bdesc + 2, kIdescI8);
              mma_i8_acc(dt, adesc0 + 4, bdesc + 4, kIdescI8);
              mma_i8_acc(dt, adesc0 + 6, bdesc + 6, kIdescI8);
            }
            mma_commit(ae0 + 8 * as);
          }
          if (ok) mma_commit(be0 + 8 * ws);
        }
        if (ok) mma_commit(accf);
      }
      mma_commit(drain);  // arrives once every MMA issued above has completed
    }
  } else if (warp >= 2 && warp <= 5) {  // epilogue warps 2..5: TMEM lane quarter (warp & 3)
    const int q = warp & 3;
    int it = 0;
    for (int t = blockIdx.x; t < p.ntiles; t += gridDim.x, ++it) {
      int z, tm, tn;
      tile_coords(p, t, z, tm, tn);
      const int m0 = tm * BM, n0 = tn * BN;
      // the tile's MMAs run before this wait ends: poll with back-off
      const bool ok = __all_sync(0xffffffffu, mbar_wait_backoff(accf, it & 1, ab, kWaitNs, 256));
      if (!ok) {
        if (lane == 0) oz_abort(ctrl, p.error, 45);
        break;
      }
      fence_after_sync();
      const int row = m0 + q * 32 + lane;
      double acc[BN];
#pragma unroll
      for (int c = 0; c < BN; ++c) acc[c] = 0.0;
      double scale = 1.0 / 16384.0;  // 2^-7g for g = 2
      for (int g = 0; g < ns; ++g, scale *= 1.0 / 128.0) {
        int v[BN];
        const uint32_t ta = tmem + (uint32_t)(g * BN) + ((uint32_t)(q * 32) << 16);
        tmem_ld32_i32_nowait(ta, v);
        tmem_ld32_i32_nowait(ta + 32, v + 32);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (g == ns - 1) {
          // every accumulator of this tile is in registers: the MMA issuer may
          // start the next tile
          fence_before_sync();
          __syncwarp();
          if (lane == 0) mbar_arrive(tmem_empty);
        }
#pragma unroll
        for (int c = 0; c < BN; ++c) acc[c] = fma((double)v[c], scale, acc[c]);
      }
      // scale by 2^(ea + eb) in one step (no intermediate underflow): for a
      // normal power of two the product with 2^e built from its exponent bits
      // is exactly ldexp (one rounding, only for a subnormal result); other
      // exponents take ldexp itself.  Lane c holds the exponents of columns
      // c and c + 32.  Each thread stores its own row in 16-byte pieces (the
      // shared memory holds the operand rings).
      const int ea = row < p.m ? p.a_exp[(long long)z * p.m + row] : 0;
      const int* eb = p.b_exp + (long long)z * p.n;
      const int eb_lo = n0 + lane < p.n ? eb[n0 + lane] : 0;
      const int eb_hi = n0 + 32 + lane < p.n ? eb[n0 + 32 + lane] : 0;
      double* out = p.c + (long long)z * p.c_mol_stride + (long long)row * p.ldc + n0;
      const bool full_row = row < p.m && n0 + BN <= p.n &&
                            ((reinterpret_cast<uintptr_t>(out) & 15) == 0);
#pragma unroll
      for (int c = 0; c < BN; c += 2) {
        double x2[2];
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int col = c + e;
          const int ex = ea + __shfl_sync(0xffffffffu, col < 32 ? eb_lo : eb_hi, col & 31);
          double x = acc[col];
          if (ex >= -1022 && ex <= 1023)
            x *= __longlong_as_double((long long)(ex + 1023) << 52);
          else
            x = ldexp(x, ex);
          x2[e] = x;
        }
        if (full_row) {
          *reinterpret_cast<double2*>(out + c) = make_double2(x2[0], x2[1]);
        } else if (row < p.m) {
          if (n0 + c < p.n) out[c] = x2[0];
          if (n0 + c + 1 < p.n) out[c + 1] = x2[1];
        }
        if (p.sym && row < p.m) {
          // the mirror C[col][row] of an element above the diagonal (a warp
          // writes 32 consecutive rows of that column); tiles below the
          // diagonal are never computed
          double* mir = p.c + (long long)z * p.c_mol_stride + row;
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            const int col = n0 + c + e;
            if (col < p.n && col > row) mir[(long long)col * p.ldc] = x2[e];
          }
        }
      }
    }
    fence_before_sync();
  }

  __syncthreads();
  if (tid == 0) {
    // every issued MMA has completed before TMEM is released; on an abort also
    // wait (bounded) for the copies still in flight
    int never = 0;
    mbar_wait_for(drain, 0, &never, kWaitNs);
    if (oz_aborted(ctrl)) {
      for (int g = ctrl->b_consumed; g < ctrl->b_issued; ++g)
        mbar_wait_for(bf0 + 8 * (g % kWRing), (g / kWRing) & 1, &never, kWaitNs);
      for (int g = ctrl->a_consumed; g < ctrl->a_issued; ++g)
        mbar_wait_for(af0 + 8 * (g % kARing), (g / kARing) & 1, &never, kWaitNs);
    }
  }
  __syncthreads();
  if (warp == 0) {
    fence_after_sync();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols)
                 : "memory");
  }
}

// rows of src (FP64, optionally times a per-column power-of-two scale) ->
// ns int8 slices and the row exponent; one warp per row
__global__ void slice_rows_kernel(const double* __restrict__ src, int nmol, long long rows, int cols,
                                  long long ld, long long mol_stride, const double* __restrict__ col_scale,
                                  int ns, int8_t* __restrict__ dst, int ldd, int* __restrict__ exps) {
  const long long nwarps = (long long)gridDim.x * (blockDim.x >> 5);
  const int lane = threadIdx.x & 31;
  for (long long gr = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
       gr < (long long)nmol * rows; gr += nwarps) {
    const long long z = gr / rows, r = gr - z * rows;
    const double* x = src + z * mol_stride + r * ld;
    const double* sc = col_scale ? col_scale + z * cols : nullptr;
    double mx = 0.0;
    for (int c = lane; c < cols; c += 32) mx = fmax(mx, fabs(sc ? x[c] * sc[c] : x[c]));
#pragma unroll
    for (int o = 16; o; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    int e = 0;
    if (mx > 0.0) frexp(mx, &e);  // mx < 2^e
    const double inv = ldexp(1.0, -e);
    int8_t* d = dst + (z * ns * rows + r) * (long long)ldd;
    const long long sstride = rows * (long long)ldd;
    for (int c = lane; c < cols; c += 32) {
      double y = (sc ? x[c] * sc[c] : x[c]) * inv;
      for (int s = 0; s < ns; ++s) {
        y *= 128.0;
        const double a = fmin(127.0, fmax(-127.0, rint(y)));
        y -= a;
        d[s * sstride + c] = (int8_t)(int)a;
      }
    }
    if (lane == 0) exps[z * rows + r] = e;
  }
}

// [batch][rows][ld] int8 read as (k < kext, row < rows, batch) boxes of 128 x box_rows
int make_map_i8(CUtensorMap* tm, const int8_t* base, int kext, int ld, long long rows, int batch,
                int box_rows) {
  auto enc = encode_fn();
  if (!enc) return fail(VQC_STATUS_CUDA_ERROR, "cuTensorMapEncodeTiled unavailable");
  if ((reinterpret_cast<uintptr_t>(base) & 15) || (ld % 16) || kext > ld)
    return fail(VQC_STATUS_INVALID_ARGUMENT, "ozaki tensor map: alignment/stride");
  cuuint64_t dims[3] = {(cuuint64_t)kext, (cuuint64_t)rows, (cuuint64_t)batch};
  cuuint64_t strides[2] = {(cuuint64_t)ld, (cuuint64_t)ld * (cuuint64_t)rows};
  cuuint32_t box[3] = {(cuuint32_t)BKB, (cuuint32_t)box_rows, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = enc(tm, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<int8_t*>(base), dims, strides,
                   box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(VQC_STATUS_CUDA_ERROR, "cuTensorMapEncodeTiled failed (int8)");
  return VQC_STATUS_SUCCESS;
}

}  // namespace oz
}  // namespace vqc

using namespace vqc;

extern "C" int vqc_ozaki_slice_rows(const double* src, int32_t nmol, int64_t rows, int32_t cols,
                                    int64_t ld, int64_t mol_stride, const double* col_scale,
                                    int32_t nslices, int8_t* dst, int32_t ldd, int32_t* exps,
                                    void* stream) {
  if (!src || !dst || !exps || nmol <= 0 || rows <= 0 || cols <= 0 || ld < cols || ldd < cols ||
      nslices < 1 || nslices > oz::kMaxSlices)
    return fail(VQC_STATUS_INVALID_ARGUMENT, "ozaki_slice_rows: bad argument");
  const long long total = (long long)nmol * rows;
  const long long blocks = std::min<long long>((total + 7) / 8, 148LL * 64);
  oz::slice_rows_kernel<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(
      src, nmol, rows, cols, ld, mol_stride, col_scale, nslices, dst, ldd, exps);
  count_launch();
  return cuda_status(cudaGetLastError(), "ozaki_slice_rows");
}

extern "C" int vqc_ozaki_gemm(const int8_t* a_slices, const int32_t* a_exps, int64_t m,
                              const int8_t* b_slices, const int32_t* b_exps, int32_t n, int32_t k,
                              int32_t ldk, int32_t nmol, int32_t nslices, int32_t upper, double* c,
                              int64_t ldc, int64_t c_mol_stride, int32_t* error, void* stream) {
  if (!a_slices || !a_exps || !b_slices || !b_exps || !c || m <= 0 || n <= 0 || k <= 0 ||
      ldk < k || ldk % 16 || nmol <= 0 || nslices < 1 || nslices > oz::kMaxSlices || ldc < n ||
      upper < 0 || upper > 2 ||
      m > 0x7fffffffLL || (long long)k * nslices * 16129LL > 0x7fffffffLL ||
      (long long)nmol * nslices > 0x7fffffffLL || (m + oz::BM - 1) / oz::BM > 65535 || nmol > 65535)
    return fail(VQC_STATUS_INVALID_ARGUMENT, "ozaki_gemm: bad argument");
  CUtensorMap ta, tb;
  int st = oz::make_map_i8(&ta, a_slices, k, ldk, m, nmol * nslices, oz::BM);
  if (!st) st = oz::make_map_i8(&tb, b_slices, k, ldk, n, nmol * nslices, oz::BN);
  if (st) return st;
  oz::OzParams p{};
  p.m = (int)m;
  p.n = n;
  p.k = k;
  p.ns = nslices;
  p.upper = upper == 1 ? 1 : 0;
  p.sym = upper == 2 ? 1 : 0;
  if (p.sym && (m != n || a_slices != b_slices || a_exps != b_exps))
    return fail(VQC_STATUS_INVALID_ARGUMENT, "ozaki_gemm: symmetric output needs A == B");
  p.ntn = (n + oz::BN - 1) / oz::BN;
  p.ntm = (int)((m + oz::BM - 1) / oz::BM);
  long long per = (long long)p.ntn * p.ntm;
  if (p.sym) {
    per = 0;
    for (int tm = 0; tm < p.ntm; ++tm) per += std::max(0, p.ntn - 2 * tm);
  }
  p.sym_per = (int)per;
  const long long ntiles = per * nmol;
  if (ntiles > 0x7fffffffLL) return fail(VQC_STATUS_INVALID_ARGUMENT, "ozaki_gemm: too many tiles");
  p.ntiles = (int)ntiles;
  p.a_exp = a_exps;
  p.b_exp = b_exps;
  p.c = c;
  p.ldc = ldc;
  p.c_mol_stride = c_mol_stride;
  p.error = error;
  cudaError_t e = cudaFuncSetAttribute(oz::ozaki_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       oz::SMEM);
  if (e != cudaSuccess) return cuda_status(e, "ozaki smem attribute");
  const int sms = vqc::tc::sm_count();
  const int ctas = p.ntiles < sms ? p.ntiles : sms;  // persistent: one CTA per SM
  oz::ozaki_gemm_kernel<<<ctas, oz::kThreads, oz::SMEM, (cudaStream_t)stream>>>(ta, tb, p);
  count_launch();
  return cuda_status(cudaGetLastError(), "ozaki_gemm");
}
