// Split-precision (3xTF32) tensor-core GEMMs for the mixed-precision exchange.
//
// Products are formed on the 5th-generation tensor cores (tcgen05.mma
// kind::tf32, M = 128, accumulator in TMEM) as
//     A B^T = A_hi B_hi^T + A_hi B_lo^T + A_lo B_hi^T,
// x_hi = rn_tf32(x), x_lo = rn_tf32(x - x_hi): round-to-nearest splitting, so
// the products carry ~2^-22 relative error without the one-sided bias of
// truncation.  The streamed B tile of the half transform is the exception:
// the MMA reads its FP32 values, whose TF32 truncation is x_hi, and
// x_lo = rn_tf32(x - x_hi) (exact residual, rounded to nearest) carries the
// rest, so the split stays unbiased (~2^-22 per element) without writing x_hi
// back.  Operand tiles arrive by TMA (128-byte swizzle, K-major).
//
//   half_ws_kernel -- U[mol][mu][Q][i] = sum_nu B[mol][mu][Q][nu] C[nu][i]
//     (reference src/scf/cuda/df_occupied_exchange.cpp:251-257).  Persistent
//     over (mu, 128-row Q tile) items; each CTA takes a contiguous item range
//     with mu fastest, so rho rows accumulate in registers across items.  U is
//     written as [mol][mu][i][Q] (Q contiguous: coalesced epilogue stores).
//     Warp roles: one TMA producer, eight splitter warps that write the
//     streamed FP32 B tile's lo part into a sibling buffer, one
//     MMA-issuing thread, eight epilogue warps (two per TMEM lane quarter).
//     C arrives pre-split.  Two TMEM accumulators let an item's epilogue (U
//     written already split, rho[Q] += 2 sum_i U C[mu][i] for J) overlap the next
//     item's MMAs.  The kernel streams B once: HBM-bound by design.
//   gram_ws_kernel -- K[mol] += U U^T over kdim = X * o_pad (reference
//     df_occupied_exchange.cpp:262-279) from the pre-split U: a pure
//     TMA -> MMA pipeline over upper-triangle 128x128 tiles and split K
//     ranges.  The symmetric two-operand form K += A B^T + B A^T (two K
//     segments, operands swapped in the second) serves the incremental
//     exchange K(D) = K(D0) + 2 (V dU^T + dU V^T) about an FP64 anchor.  The tensor core's FP32 accumulation is not round-to-nearest
//     (about 2^-24 relative bias per accumulation step), so chains are kept to
//     kGramFlush K-blocks and drained into FP64 registers by eight epilogue
//     warps (double-buffered TMEM); tiles add FP64 partials (and the mirror
//     of off-diagonal tiles) into the output.
//
// Every mbarrier wait is bounded by a 2 s %globaltimer budget; on expiry the
// CTA records an error code, every role stops issuing work, thread 0 waits
// (bounded) for the copies and MMAs it has in flight, TMEM is freed and the
// kernel returns.
#include <cuda.h>
#include <cudaTypedefs.h>

#include "tc_common.cuh"
#include "vqc_df.h"
#include "vqc_plan.hpp"

namespace vqc {
namespace tc {

constexpr int BM = 128;
constexpr int BK = 32;  // FP32 elements per K-block: one 128-byte swizzle row
template <int BN>
__device__ __forceinline__ constexpr uint32_t instr_desc() {
  // D = F32 (bits 4-5 = 1), A = B = TF32 (2), both K-major, N >> 3, M >> 4
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(BN >> 3) << 17) |
         ((uint32_t)(BM >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                         uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// accumulate into D (no predicate to set up)
__device__ __forceinline__ void mma_tf32_acc(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                             uint32_t idesc) {
  asm volatile("tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, 1;" ::"r"(tmem_d), "l"(adesc),
               "l"(bdesc), "r"(idesc)
               : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
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
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Round a finite FP32 value to the nearest TF32 value (10 mantissa bits),
// ties away from zero: add half of the dropped 13-bit field to the
// sign-magnitude bit pattern (a carry moves into the exponent as it should)
// and clear the field.  Two integer ops on the full-rate ALUs instead of the
// narrower conversion pipe; same result as cvt.rna.tf32.f32 for finite x.
__device__ __forceinline__ float rn_tf32(float x) {
  return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
}

// x with its 13 low mantissa bits cleared: the TF32 value the tensor core
// takes from an FP32 operand; x - tf32_trunc(x) is exact in FP32
__device__ __forceinline__ float tf32_trunc(float x) {
  return __uint_as_float(__float_as_uint(x) & 0xFFFFE000u);
}


// Shared control block behind the operand stages.
struct Ctrl {
  uint64_t full[4], conv[4], empty[4], acc_full[2], acc_empty[2];
  uint32_t tmem;
  int abort;
  int issued;    // k-steps the producer issued
  int consumed;  // k-steps whose operands have been taken over (full barrier passed)
  int commits;   // MMA commits to empty barriers
};

__device__ __forceinline__ void set_abort(Ctrl* c, int* error, int code) {
  if (error) atomicExch(error, code);
  *reinterpret_cast<volatile int*>(&c->abort) = 1;
}

__device__ __forceinline__ bool aborted(Ctrl* c) {
  return *reinterpret_cast<volatile int*>(&c->abort) != 0;
}

// ---------------------------------------------------------------------------
// half transform: U[z][Q][i] = sum_nu B[z][Q][nu] C[mol(z)][i][nu], 3xTF32,
// persistent over (z, 128-row Q tile) items; warp roles:
//   w0 TMA producer, w1-w8 splitters (A -> lo; the MMA reads A_hi as the TF32
//   truncation of the FP32 tile), w9 MMA issuer,
//   w10-w17 epilogue (TMEM -> U hi/lo in HBM, rho partial sums)
// ---------------------------------------------------------------------------

// warps: 0 TMA producer, 1-8 splitters, 9 MMA issuer, 10-17 epilogue (two per
// TMEM lane quarter, interleaved 16-column chunks): the split and the
// TMEM -> HBM epilogue are per-warp latency-bound, so each has eight warps
#ifndef VQC_HALF_SPLIT_WARPS
#define VQC_HALF_SPLIT_WARPS 8
#endif
#ifndef VQC_HALF_EPI_WARPS
#define VQC_HALF_EPI_WARPS 8
#endif
constexpr int kSplitWarps = VQC_HALF_SPLIT_WARPS;
constexpr int kEpiWarps = VQC_HALF_EPI_WARPS;  // a multiple of 4 (TMEM lane quarters)
constexpr int kEpiGroups = kEpiWarps / 4;      // warps sharing one lane quarter
constexpr int kMmaWarp = 1 + kSplitWarps;
constexpr int kEpiWarp0 = kMmaWarp + 1;
constexpr int kHalfThreads = 32 * (kEpiWarp0 + kEpiWarps);
static_assert(kEpiWarps % 4 == 0 && kEpiWarps >= 4, "epilogue warps per lane quarter");
constexpr int kGramThreads = 320;
constexpr int kTmemBuf = 128;  // columns per accumulator buffer (two buffers)

template <int BN>
struct HalfCfg {
  static constexpr int A_BYTES = BM * BK * 4;
  static constexpr int C_BYTES = BN * BK * 4;
  static constexpr int STAGE = 2 * A_BYTES + 2 * C_BYTES;
  static constexpr int S = (214 * 1024) / STAGE >= 4 ? 4 : (214 * 1024) / STAGE;
  static constexpr int SMEM = S * STAGE + 1024 + (int)sizeof(Ctrl) + 64;
  // TMEM columns per accumulator buffer: [0, BN) takes A_hi C_hi + A_lo C_hi,
  // [BN, 2 BN) takes A_hi C_lo (one N = 2 BN MMA over the adjacent C_hi, C_lo
  // tiles); allocations are powers of two
  static constexpr int TBUF = 2 * BN <= 128 ? 128 : 256;
  static_assert(BN % 16 == 0 && BN >= 16 && 2 * BN <= 256, "BN");
  static_assert(S >= 2, "pipeline");
};

struct HalfParams {
  int nao, naux, nocc, ldq, nitems, nqt, nk, per_cta;
  float* u_hi;
  float* u_lo;
  double* rho;
  const double* cvec;
  const double* dens;  // optional D[mol][mu][nu]: the splitters also form rho_dens
  double* rho_dens;    // rho_dens[mol][Q] += sum_{mu,nu} B[mu][Q][nu] D[mu][nu] (FP64)
  int* error;
};

template <int BN>
__global__ void __launch_bounds__(kHalfThreads, 1)
    half_ws_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmCh,
                   const __grid_constant__ CUtensorMap tmCl, HalfParams p) {
  using C = HalfCfg<BN>;
  constexpr int S = C::S;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  Ctrl* ctrl = reinterpret_cast<Ctrl*>(smem + S * C::STAGE);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t full0 = smem_u32(ctrl->full), conv0 = smem_u32(ctrl->conv);
  const uint32_t empty0 = smem_u32(ctrl->empty), af0 = smem_u32(ctrl->acc_full);
  const uint32_t ae0 = smem_u32(ctrl->acc_empty);
  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(full0 + 8 * s, 1);
      mbar_init(conv0 + 8 * s, kSplitWarps);
      mbar_init(empty0 + 8 * s, 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(af0 + 8 * b, 1);
      mbar_init(ae0 + 8 * b, kEpiWarps);
    }
    ctrl->abort = 0;
    ctrl->issued = ctrl->consumed = ctrl->commits = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&ctrl->tmem)),
                 "r"(2 * C::TBUF)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = ctrl->tmem;
  auto stage = [&](int s) { return smem + s * C::STAGE; };
  const int nk = p.nk;
  volatile int* ab = &ctrl->abort;

  if (warp == 0) {
    if (lane == 0) {  // producer
      int g = 0;
      const int i0 = blockIdx.x * p.per_cta, i1 = min(p.nitems, i0 + p.per_cta);
      for (int item = i0; item < i1 && !aborted(ctrl); ++item) {
        const int mu = item % p.nao, qt = (item / p.nao) % p.nqt, mol = item / (p.nao * p.nqt);
        const int z = mol * p.nao + mu;
        for (int kb = 0; kb < nk; ++kb, ++g) {
          const int s = g % S;
          if (g >= S && !mbar_wait(empty0 + 8 * s, ((g / S) - 1) & 1, ab)) {
            set_abort(ctrl, p.error, 11);
            break;
          }
          const uint32_t a = smem_u32(stage(s));
          mbar_expect_tx(full0 + 8 * s, C::A_BYTES + 2 * C::C_BYTES);
          tma_load_3d(a, &tmA, kb * BK, qt * BM, z, full0 + 8 * s);
          tma_load_3d(a + 2 * C::A_BYTES, &tmCh, kb * BK, 0, mol, full0 + 8 * s);
          tma_load_3d(a + 2 * C::A_BYTES + C::C_BYTES, &tmCl, kb * BK, 0, mol, full0 + 8 * s);
          *reinterpret_cast<volatile int*>(&ctrl->issued) = g + 1;
        }
      }
    }
  } else if (warp >= 1 && warp <= kSplitWarps) {  // splitters
    const int ts = tid - 32;
    int g = 0;
    const int i0 = blockIdx.x * p.per_cta, i1 = min(p.nitems, i0 + p.per_cta);
    // With p.dens the splitters also form the fitted density from the exact
    // FP32 values they split: rho_dens[Q] += sum_nu B[mu][Q][nu] D[mu][nu],
    // four-term FP32 partial sums accumulated in FP64 (relative error ~2^-23
    // of sum |B D|; only the tensor-core phase before the FP64 anchor uses
    // it).  Float4 k of a 128-byte-swizzled stage holds row r = k / 8 and
    // logical chunk (k % 8) ^ (r % 8); this thread's rows are ts / 8 + 32 i
    // (i < 4), all in the same chunk, so its four nu are fixed per K-block and
    // the eight lanes sharing a row cover its 32 columns.
    static_assert((C::A_BYTES / 16) % (32 * kSplitWarps) == 0 && kSplitWarps % 2 == 0,
                  "each splitter thread owns whole float4 rows in one swizzle chunk");
    constexpr int kRowsPerThread = C::A_BYTES / 16 / (32 * kSplitWarps);
    const int chunk = (ts & 7) ^ ((ts >> 3) & 7);
    double racc[kRowsPerThread];
#pragma unroll
    for (int i = 0; i < kRowsPerThread; ++i) racc[i] = 0.0;
    int rkey = -1;
    // density weights D[mol][mu][nu] of (item, K-block): this thread's four nu
    auto load_weights = [&](int it, int kb, double (&w)[4]) {
      w[0] = w[1] = w[2] = w[3] = 0.0;
      if (!p.dens || it >= i1) return;
      const int m = it % p.nao, key = it / p.nao;
      const double* drow = p.dens + ((size_t)(key / p.nqt) * p.nao + m) * p.nao;
      const int nu = kb * BK + 4 * chunk;
#pragma unroll
      for (int e = 0; e < 4; ++e)
        if (nu + e < p.nao) w[e] = __ldg(drow + nu + e);
    };
    double wn[4];
    load_weights(i0, 0, wn);
    for (int item = i0; item < i1; ++item) {
      const int mu = item % p.nao, key = item / p.nao;  // key = mol * nqt + qt
      if (p.dens && key != rkey) {
        if (rkey >= 0) {
#pragma unroll
          for (int i = 0; i < kRowsPerThread; ++i) {
            double v = racc[i];
            v += __shfl_xor_sync(0xffffffffu, v, 1);
            v += __shfl_xor_sync(0xffffffffu, v, 2);
            v += __shfl_xor_sync(0xffffffffu, v, 4);
            const int qrow = (rkey % p.nqt) * BM + (ts >> 3) + 32 * kSplitWarps / 8 * i;
            if ((ts & 7) == 0 && qrow < p.naux)
              atomicAdd(p.rho_dens + (size_t)(rkey / p.nqt) * p.naux + qrow, v);
            racc[i] = 0.0;
          }
        }
        rkey = key;
      }
      (void)mu;
      for (int kb = 0; kb < nk; ++kb, ++g) {
        const int s = g % S;
        // this K-block's density weights were loaded one step ahead (kept in
        // FP64 until here so no conversion waits on the load); fetch the next
        // step's now, before the barrier wait hides their latency
        const float w0 = (float)wn[0], w1 = (float)wn[1], w2 = (float)wn[2], w3 = (float)wn[3];
        if (kb + 1 < nk) load_weights(item, kb + 1, wn);
        else load_weights(item + 1, 0, wn);
        // every lane waits; the warp leaves together (no lane may skip a
        // later warp-collective alone)
        if (!__all_sync(0xffffffffu, mbar_wait(full0 + 8 * s, (g / S) & 1, ab))) {
          if (lane == 0) set_abort(ctrl, p.error, 12);
          goto split_done;
        }
        if (ts == 0) *reinterpret_cast<volatile int*>(&ctrl->consumed) = g + 1;
        // the FP32 tile stays in place: the MMA takes its TF32 truncation as
        // A_hi, and the splitters write A_lo = rn_tf32(x - tf32_trunc(x))
        const float4* a = reinterpret_cast<const float4*>(stage(s));
        float4* alo = reinterpret_cast<float4*>(stage(s) + C::A_BYTES);
#pragma unroll
        for (int i = 0; i < kRowsPerThread; ++i) {
          const int k = ts + i * 32 * kSplitWarps;
          const float4 v = a[k];
          if (p.dens)
            racc[i] += (double)fmaf(v.x, w0, fmaf(v.y, w1, fmaf(v.z, w2, v.w * w3)));
          float4 lo;
          lo.x = rn_tf32(v.x - tf32_trunc(v.x));
          lo.y = rn_tf32(v.y - tf32_trunc(v.y));
          lo.z = rn_tf32(v.z - tf32_trunc(v.z));
          lo.w = rn_tf32(v.w - tf32_trunc(v.w));
          alo[k] = lo;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncwarp();
        if (lane == 0) mbar_arrive(conv0 + 8 * s);
      }
    }
    if (p.dens && rkey >= 0) {
#pragma unroll
      for (int i = 0; i < kRowsPerThread; ++i) {
        double v = racc[i];
        v += __shfl_xor_sync(0xffffffffu, v, 1);
        v += __shfl_xor_sync(0xffffffffu, v, 2);
        v += __shfl_xor_sync(0xffffffffu, v, 4);
        const int qrow = (rkey % p.nqt) * BM + (ts >> 3) + 32 * kSplitWarps / 8 * i;
        if ((ts & 7) == 0 && qrow < p.naux)
          atomicAdd(p.rho_dens + (size_t)(rkey / p.nqt) * p.naux + qrow, v);
      }
    }
  split_done:;
  } else if (warp == kMmaWarp) {
    if (lane == 0) {  // MMA issuer
      constexpr uint32_t idesc = instr_desc<BN>(), idesc2 = instr_desc<2 * BN>();
      int g = 0, t = 0;
      const int i0 = blockIdx.x * p.per_cta, i1 = min(p.nitems, i0 + p.per_cta);
      for (int item = i0; item < i1 && !aborted(ctrl); ++item, ++t) {
        const int b = t & 1;
        if (t >= 2 && !mbar_wait(ae0 + 8 * b, ((t >> 1) - 1) & 1, ab)) {
          set_abort(ctrl, p.error, 13);
          break;
        }
        fence_after_sync();
        const uint32_t dt = tmem + b * C::TBUF;
        bool ok = true;
        for (int kb = 0; kb < nk; ++kb, ++g) {
          const int s = g % S;
          if (!mbar_wait(conv0 + 8 * s, (g / S) & 1, ab)) {
            set_abort(ctrl, p.error, 14);
            ok = false;
            break;
          }
          fence_after_sync();
          // descriptors advance by (byte offset >> 4) in their address field
          const uint32_t ahi = smem_u32(stage(s));
          const uint64_t dahi = smem_desc(ahi), dalo = smem_desc(ahi + C::A_BYTES);
          // C_lo directly follows C_hi (C_BYTES = BN rows of 128 bytes), so one
          // descriptor spans both as a 2 BN-row operand
          const uint64_t dchi = smem_desc(ahi + 2 * C::A_BYTES);
          const uint32_t acc0 = kb == 0 ? 0u : 1u;
#pragma unroll
          for (int kk = 0; kk < BK / 8; ++kk) {
            const uint64_t off = (uint64_t)kk * 2;  // 32 bytes per K-step
            if (kk == 0) mma_tf32(dt, dahi + off, dchi + off, idesc2, acc0);
            else mma_tf32_acc(dt, dahi + off, dchi + off, idesc2);
            mma_tf32_acc(dt, dalo + off, dchi + off, idesc);
          }
          mma_commit(empty0 + 8 * s);
          *reinterpret_cast<volatile int*>(&ctrl->commits) = g + 1;
        }
        if (!ok) break;
        mma_commit(af0 + 8 * b);
      }
    }
  } else {  // epilogue warps kEpiWarp0 .. kEpiWarp0 + kEpiWarps - 1
    const int q = warp & 3;  // TMEM lane quarter this warp may access
    const int half = (warp - kEpiWarp0) >> 2;  // which interleaved 16-column chunks
    int t = 0;
    const int i0 = blockIdx.x * p.per_cta, i1 = min(p.nitems, i0 + p.per_cta);
    double rho_acc = 0.0;
    int rho_key = -1;  // (mol, qt) whose rho rows rho_acc belongs to
    for (int item = i0; item < i1; ++item, ++t) {
      const int b = t & 1;
      const int mu = item % p.nao, key = item / p.nao;  // key = mol * nqt + qt
      const int qt = key % p.nqt, mol = key / p.nqt;
      const int z = mol * p.nao + mu;
      const int row = qt * BM + q * 32 + lane;
      const bool valid = row < p.naux;
      if (key != rho_key) {
        if (rho_key >= 0) {
          const int prow = (rho_key % p.nqt) * BM + q * 32 + lane;
          if (prow < p.naux && p.rho)
            atomicAdd(p.rho + (size_t)(rho_key / p.nqt) * p.naux + prow, 2.0 * rho_acc);
        }
        rho_acc = 0.0;
        rho_key = key;
      }
      if (!__all_sync(0xffffffffu, mbar_wait(af0 + 8 * b, (t >> 1) & 1, ab))) {
        if (lane == 0) set_abort(ctrl, p.error, 15);
        break;
      }
      fence_after_sync();
      // U[z][i][Q]: lanes run along Q, so every store is one coalesced 128-byte row
      float* uh = p.u_hi + (size_t)z * p.nocc * p.ldq + row;
      float* ul = p.u_lo + (size_t)z * p.nocc * p.ldq + row;
      const double* cv = p.cvec + (size_t)z * p.nocc;
#pragma unroll
      for (int c = 16 * half; c < BN; c += 16 * kEpiGroups) {
        float v[16], w[16];
        const uint32_t tb = tmem + b * C::TBUF + ((uint32_t)(q * 32) << 16) + c;
        tmem_ld16(tb, v);
        tmem_ld16(tb + BN, w);
#pragma unroll
        for (int k = 0; k < 16; ++k) v[k] += w[k];
        if (valid) {
#pragma unroll
          for (int k = 0; k < 16; ++k) {
            const int col = c + k;
            if (col < p.nocc) {
              const float h = rn_tf32(v[k]);
              uh[(size_t)col * p.ldq] = h;
              ul[(size_t)col * p.ldq] = rn_tf32(v[k] - h);
              if (p.rho) rho_acc += (double)v[k] * __ldg(cv + col);
            }
          }
        }
      }
      fence_before_sync();
      __syncwarp();
      if (lane == 0) mbar_arrive(ae0 + 8 * b);
    }
    if (rho_key >= 0 && !aborted(ctrl)) {
      const int prow = (rho_key % p.nqt) * BM + q * 32 + lane;
      if (prow < p.naux && p.rho)
        atomicAdd(p.rho + (size_t)(rho_key / p.nqt) * p.naux + prow, 2.0 * rho_acc);
    }
  }

  fence_before_sync();
  __syncthreads();
  if (aborted(ctrl) && tid == 0) {
    // bounded drain of copies and MMAs still in flight
    int never = 0;
    const int issued = ctrl->issued, consumed = ctrl->consumed;
    for (int g = consumed; g < issued; ++g)
      mbar_wait(full0 + 8 * (g % S), (g / S) & 1, &never);
    if (ctrl->commits > 0) {
      const int lc = ctrl->commits - 1;
      mbar_wait(empty0 + 8 * (lc % S), (lc / S) & 1, &never);
    }
  }
  __syncthreads();
  if (warp == 0) {
    fence_after_sync();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(2 * C::TBUF)
                 : "memory");
  }
}

// ---------------------------------------------------------------------------
// Gram product: K[z] += U U^T over kdim with pre-split U (hi, lo) in HBM;
// upper-triangle 128x128 tiles, split K range; warp roles:
//   w0 TMA producer, w1 MMA issuer, w2-w9 epilogue (two column halves per
//   TMEM lane quarter; FP64 accumulators drained every kGramFlush K-blocks)
// ---------------------------------------------------------------------------

constexpr int kGramFlush = 4;  // K-blocks per FP32 TMEM chain before the FP64 drain (48 accumulation steps)

struct GramCfg {
  static constexpr int TILE = BM * BK * 4;  // 16 KB
  static constexpr int STAGE = 4 * TILE;    // A hi, A lo, B hi, B lo
  static constexpr int S = 3;
  static constexpr int SMEM = S * STAGE + 1024 + (int)sizeof(Ctrl) + 64;
};

struct GramParams {
  int nao, kdim, ntiles_ut, nt, kblocks_per_split, ksplit;
  int nseg;  // 1: A A^T (B maps unused); 2: A B^T + B A^T
  double* kout;
  int* error;
};

__global__ void __launch_bounds__(kGramThreads, 1)
    gram_ws_kernel(const __grid_constant__ CUtensorMap tmAH, const __grid_constant__ CUtensorMap tmAL,
                   const __grid_constant__ CUtensorMap tmBH, const __grid_constant__ CUtensorMap tmBL,
                   GramParams p) {
  using C = GramCfg;
  constexpr int S = C::S;
  constexpr int BN = 128;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  Ctrl* ctrl = reinterpret_cast<Ctrl*>(smem + S * C::STAGE);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // decode (upper-triangle tile, molecule, split)
  const int tile = blockIdx.x;
  int mt = 0, rem = tile;
  while (rem >= p.nt - mt) {
    rem -= p.nt - mt;
    ++mt;
  }
  const int nt = mt + rem;
  const int z = blockIdx.y / p.ksplit, split = blockIdx.y % p.ksplit;
  const int kb_seg = (p.kdim + BK - 1) / BK;  // K-blocks per segment
  const int kb_total = kb_seg * p.nseg;
  const int kb0 = split * p.kblocks_per_split;
  const int kb1 = min(kb_total, kb0 + p.kblocks_per_split);
  const int nkb = kb1 - kb0;
  if (nkb <= 0 || mt >= p.nt) return;
  const int nchains = (nkb + kGramFlush - 1) / kGramFlush;
  // MMA width: the tile's in-range columns rounded up to 16 (M = 128 allows
  // N = 16..256 in steps of 16); TMEM columns past it are never read
  const int nmma = min(BN, (p.nao - nt * BN + 15) & ~15);
  // a diagonal tile of A A^T multiplies a row block by itself: one copy of
  // the operands serves both sides
  const bool diag = p.nseg == 1 && mt == nt;

  const uint32_t full0 = smem_u32(ctrl->full), empty0 = smem_u32(ctrl->empty);
  const uint32_t af0 = smem_u32(ctrl->acc_full), ae0 = smem_u32(ctrl->acc_empty);
  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(full0 + 8 * s, 1);
      mbar_init(empty0 + 8 * s, 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(af0 + 8 * b, 1);
      mbar_init(ae0 + 8 * b, 8);
    }
    ctrl->abort = 0;
    ctrl->issued = ctrl->consumed = ctrl->commits = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&ctrl->tmem)),
                 "r"(2 * kTmemBuf)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = ctrl->tmem;
  auto stage = [&](int s) { return smem + s * C::STAGE; };
  volatile int* ab = &ctrl->abort;
  double acc[64];
#pragma unroll
  for (int c = 0; c < 64; ++c) acc[c] = 0.0;

  if (warp == 0) {
    if (lane == 0) {  // producer
      for (int i = 0; i < nkb; ++i) {
        const int s = i % S;
        if (i >= S && !mbar_wait(empty0 + 8 * s, ((i / S) - 1) & 1, ab)) {
          set_abort(ctrl, p.error, 21);
          break;
        }
        const uint32_t a = smem_u32(stage(s));
        const int gk = kb0 + i, seg = gk / kb_seg;
        const int k = (gk - seg * kb_seg) * BK;
        // segment 0: rows mt of A against rows nt of B; segment 1 swaps them
        const bool one = p.nseg == 1;
        const CUtensorMap* rh = seg ? &tmBH : &tmAH;
        const CUtensorMap* rl = seg ? &tmBL : &tmAL;
        const CUtensorMap* ch = (one || seg) ? &tmAH : &tmBH;
        const CUtensorMap* cl = (one || seg) ? &tmAL : &tmBL;
        mbar_expect_tx(full0 + 8 * s, diag ? 2 * C::TILE : C::STAGE);
        tma_load_3d(a, rh, k, mt * BM, z, full0 + 8 * s);
        tma_load_3d(a + C::TILE, rl, k, mt * BM, z, full0 + 8 * s);
        if (!diag) {
          tma_load_3d(a + 2 * C::TILE, ch, k, nt * BN, z, full0 + 8 * s);
          tma_load_3d(a + 3 * C::TILE, cl, k, nt * BN, z, full0 + 8 * s);
        }
        *reinterpret_cast<volatile int*>(&ctrl->issued) = i + 1;
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {  // MMA issuer
      const uint32_t idesc = (instr_desc<BN>() & ~(0x3fu << 17)) | ((uint32_t)(nmma >> 3) << 17);
      int i = 0;
      for (int ch = 0; ch < nchains && !aborted(ctrl); ++ch) {
        const int b = ch & 1;
        if (ch >= 2 && !mbar_wait(ae0 + 8 * b, ((ch >> 1) - 1) & 1, ab)) {
          set_abort(ctrl, p.error, 22);
          break;
        }
        fence_after_sync();
        const uint32_t dt = tmem + b * kTmemBuf;
        const int iend = min(nkb, i + kGramFlush);
        bool ok = true;
        for (int first = i; i < iend; ++i) {
          const int s = i % S;
          if (!mbar_wait(full0 + 8 * s, (i / S) & 1, ab)) {
            set_abort(ctrl, p.error, 23);
            ok = false;
            break;
          }
          *reinterpret_cast<volatile int*>(&ctrl->consumed) = i + 1;
          fence_after_sync();
          // descriptors advance by (byte offset >> 4) in their address field
          const uint32_t ahi = smem_u32(stage(s));
          const uint64_t dahi = smem_desc(ahi), dalo = smem_desc(ahi + C::TILE);
          const uint64_t dbhi = diag ? dahi : smem_desc(ahi + 2 * C::TILE);
          const uint64_t dblo = diag ? dalo : smem_desc(ahi + 3 * C::TILE);
          const uint32_t acc0 = i == first ? 0u : 1u;
#pragma unroll
          for (int kk = 0; kk < BK / 8; ++kk) {
            const uint64_t off = (uint64_t)kk * 2;  // 32 bytes per K-step
            if (kk == 0) mma_tf32(dt, dalo + off, dbhi + off, idesc, acc0);
            else mma_tf32_acc(dt, dalo + off, dbhi + off, idesc);
            mma_tf32_acc(dt, dahi + off, dblo + off, idesc);
            mma_tf32_acc(dt, dahi + off, dbhi + off, idesc);
          }
          mma_commit(empty0 + 8 * s);
          *reinterpret_cast<volatile int*>(&ctrl->commits) = i + 1;
        }
        if (!ok) break;
        mma_commit(af0 + 8 * b);
      }
    }
  } else {  // epilogue warps 2..9
    const int q = warp & 3, half = (warp - 2) >> 2;
    for (int ch = 0; ch < nchains; ++ch) {
      const int b = ch & 1;
      if (!__all_sync(0xffffffffu, mbar_wait(af0 + 8 * b, (ch >> 1) & 1, ab))) {
        if (lane == 0) set_abort(ctrl, p.error, 24);
        break;
      }
      fence_after_sync();
#pragma unroll
      for (int c = 0; c < 64; c += 16) {
        if (half * 64 + c >= nmma) continue;  // warp-uniform
        float v[16];
        tmem_ld16(tmem + b * kTmemBuf + half * 64 + c + ((uint32_t)(q * 32) << 16), v);
#pragma unroll
        for (int k = 0; k < 16; ++k) acc[c + k] += (double)v[k];
      }
      fence_before_sync();
      __syncwarp();
      if (lane == 0) mbar_arrive(ae0 + 8 * b);
    }
    if (!aborted(ctrl)) {
      const int row = mt * BM + q * 32 + lane;
      if (row < p.nao) {
        double* base = p.kout + (size_t)z * p.nao * p.nao;
#pragma unroll
        for (int c = 0; c < 64; ++c) {
          const int col = nt * BN + half * 64 + c;
          if (col < p.nao) {
            atomicAdd(base + (size_t)row * p.nao + col, acc[c]);
            if (mt != nt) atomicAdd(base + (size_t)col * p.nao + row, acc[c]);
          }
        }
      }
    }
  }

  fence_before_sync();
  __syncthreads();
  if (aborted(ctrl) && tid == 0) {
    int never = 0;
    const int issued = ctrl->issued, consumed = ctrl->consumed;
    for (int g = consumed; g < issued; ++g)
      mbar_wait(full0 + 8 * (g % S), (g / S) & 1, &never);
    if (ctrl->commits > 0) {
      const int lc = ctrl->commits - 1;
      mbar_wait(empty0 + 8 * (lc % S), (lc / S) & 1, &never);
    }
  }
  __syncthreads();
  if (warp == 0) {
    fence_after_sync();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(2 * kTmemBuf)
                 : "memory");
  }
}

// ---------------------------------------------------------------------------
// Coulomb build J[mol][mu][nu] = sum_Q B[mol][mu][Q][nu] rho[mol][Q] (nu <= mu,
// mirrored) from the FP32 aux-major tensor, streamed by TMA: persistent CTAs
// take (mol, mu) rows largest-first in round-robin order; for each 32-column
// nu chunk of the row the producer streams the 128-row Q blocks through a
// ring of kCoulStages 16 KB stages, eight consumer warps (16 Q rows each, one
// nu per lane) accumulate in FP64, and the chunk's 32 sums meet in shared
// memory.  Reference src/scf/cuda/df_coulomb.cpp:24 (FP64 cublasDgemv).
// ---------------------------------------------------------------------------

constexpr int kCoulStages = 8;
constexpr int kCoulWarps = 8;                       // consumers
constexpr int kCoulThreads = 32 * (1 + kCoulWarps);  // + producer warp
constexpr int kCoulTile = BM * BK * 4;               // 16 KB
constexpr int kCoulMaxAux = 4096;  // fitted-density entries staged in shared memory
constexpr int kCoulSmem = kCoulStages * kCoulTile + 1024 + kCoulWarps * 32 * 8 +
                          2 * kCoulStages * 8 + kCoulMaxAux * 8 + 64;

struct CoulParams {
  int nmol, nao, naux, nqt;
  const double* rho;
  double* j;
  int* error;
};

__global__ void __launch_bounds__(kCoulThreads, 1)
    coulomb_tma_kernel(const __grid_constant__ CUtensorMap tmB, CoulParams p) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  double* red = reinterpret_cast<double*>(smem + kCoulStages * kCoulTile);  // [warp][32]
  uint64_t* bars = reinterpret_cast<uint64_t*>(red + kCoulWarps * 32);
  double* srho = reinterpret_cast<double*>(bars + 2 * kCoulStages);  // [nqt * BM]
  __shared__ int abort_flag;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t full0 = smem_u32(bars), empty0 = smem_u32(bars + kCoulStages);
  if (tid == 0) {
    for (int s = 0; s < kCoulStages; ++s) {
      mbar_init(full0 + 8 * s, 1);
      mbar_init(empty0 + 8 * s, kCoulWarps);
    }
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  volatile int* ab = &abort_flag;
  const int nitems = p.nmol * p.nao;
  int issued = 0;  // producer: tiles issued

  if (warp == 0) {
    if (lane == 0) {
      int g = 0;
      bool ok = true;
      for (int it = blockIdx.x; it < nitems && ok; it += gridDim.x) {
        const int mu = p.nao - 1 - it / p.nmol, mol = it % p.nmol;
        const int nkc = mu / BK + 1;
        for (int kc = 0; kc < nkc && ok; ++kc)
          for (int qt = 0; qt < p.nqt; ++qt, ++g) {
            const int s = g % kCoulStages;
            if (g >= kCoulStages && !mbar_wait(empty0 + 8 * s, ((g / kCoulStages) - 1) & 1, ab)) {
              if (p.error) atomicExch(p.error, 51);
              *reinterpret_cast<volatile int*>(&abort_flag) = 1;
              ok = false;
              break;
            }
            mbar_expect_tx(full0 + 8 * s, kCoulTile);
            tma_load_3d(smem_u32(smem + s * kCoulTile), &tmB, kc * BK, qt * BM, mol * p.nao + mu,
                        full0 + 8 * s);
            issued = g + 1;
          }
      }
      // bounded drain of copies still in flight after an abort
      if (!ok) {
        int never = 0;
        for (int k = max(0, issued - kCoulStages); k < issued; ++k)
          mbar_wait_for(full0 + 8 * (k % kCoulStages), (k / kCoulStages) & 1, &never, kWaitNs);
      }
    }
  } else {  // consumers: warp w - 1 owns rows 16 (w - 1) .. + 15 of every tile, lane = nu
    const int cw = warp - 1;
    int g = 0;
    int rho_mol = -1;
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
      const int mu = p.nao - 1 - it / p.nmol, mol = it % p.nmol;
      const int nkc = mu / BK + 1;
      double* jm = p.j + (size_t)mol * p.nao * p.nao;
      if (mol != rho_mol) {
        // the molecule's fitted density in shared memory (zero beyond naux)
        asm volatile("bar.sync 1, %0;" ::"r"(32 * kCoulWarps) : "memory");
        for (int q = tid - 32; q < p.nqt * BM; q += 32 * kCoulWarps)
          srho[q] = q < p.naux ? __ldg(p.rho + (size_t)mol * p.naux + q) : 0.0;
        asm volatile("bar.sync 1, %0;" ::"r"(32 * kCoulWarps) : "memory");
        rho_mol = mol;
      }
      for (int kc = 0; kc < nkc; ++kc) {
        double acc4[4] = {0.0, 0.0, 0.0, 0.0};  // independent chains over the rows
        for (int qt = 0; qt < p.nqt; ++qt, ++g) {
          const int s = g % kCoulStages;
          // every consumer warp runs the same loops to the end, so all of them
          // reach each named barrier below; after an abort the waits return at once
          if (!__all_sync(0xffffffffu, mbar_wait(full0 + 8 * s, (g / kCoulStages) & 1, ab))) {
            if (lane == 0 && p.error) atomicExch(p.error, 52);
            *reinterpret_cast<volatile int*>(&abort_flag) = 1;
            continue;
          }
          const uint8_t* tile = smem + s * kCoulTile;
          const double* rq = srho + qt * BM + cw * 16;
#pragma unroll
          for (int r = 0; r < 16; ++r) {
            const int row = cw * 16 + r;  // 128-byte swizzle: chunk (lane / 4) ^ (row % 8)
            const float b = *reinterpret_cast<const float*>(
                tile + row * 128 + ((((lane >> 2) ^ (row & 7))) << 4) + ((lane & 3) << 2));
            acc4[r & 3] = fma((double)b, rq[r], acc4[r & 3]);  // rows >= naux read as zero
          }
          __syncwarp();
          if (lane == 0) mbar_arrive(empty0 + 8 * s);
        }
        red[cw * 32 + lane] = (acc4[0] + acc4[1]) + (acc4[2] + acc4[3]);
        // the consumer warps' partial sums of this chunk (named barrier over the consumers)
        asm volatile("bar.sync 1, %0;" ::"r"(32 * kCoulWarps) : "memory");
        if (cw == 0) {
          double v = 0.0;
#pragma unroll
          for (int w = 0; w < kCoulWarps; ++w) v += red[w * 32 + lane];
          const int nu = kc * BK + lane;
          if (nu <= mu && !*ab) {
            jm[(size_t)mu * p.nao + nu] = v;
            jm[(size_t)nu * p.nao + mu] = v;
          }
        }
        asm volatile("bar.sync 1, %0;" ::"r"(32 * kCoulWarps) : "memory");
      }
    }
  }
}

// Self-test of the bounded-wait error path: one warp waits on an mbarrier
// that nothing ever arrives on; the wait must give up after budget_ns and
// the kernel must report it in *error and return normally.
constexpr int kWaitSelftestCode = 31;

__global__ void wait_selftest_kernel(unsigned long long budget_ns, int* error) {
  __shared__ uint64_t bar;
  __shared__ int never;
  if (threadIdx.x == 0) {
    mbar_init(smem_u32(&bar), 1);
    never = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();
  const bool ok = mbar_wait_for(smem_u32(&bar), 0, &never, budget_ns);
  if (!__all_sync(0xffffffffu, ok) && threadIdx.x == 0) atomicExch(error, kWaitSelftestCode);
}

__global__ void split_tf32_kernel(const float* __restrict__ x, float* __restrict__ hi,
                                  float* __restrict__ lo, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const float h = rn_tf32(x[i]);
    hi[i] = h;
    lo[i] = rn_tf32(x[i] - h);
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

// 3-D FP32 tensor [batch][rows][ld] read as (k < kext, row < rows, batch) boxes of
// BK x box_rows; elements with k >= kext or row >= rows read as zero.
static int make_map(CUtensorMap* tm, const float* base, int kext, int ld, int rows, int batch,
                    int box_rows) {
  auto enc = encode_fn();
  if (!enc) return fail(VQC_STATUS_CUDA_ERROR, "cuTensorMapEncodeTiled unavailable");
  if ((reinterpret_cast<uintptr_t>(base) & 15) || (ld % 4) || kext > ld || box_rows > 256)
    return fail(VQC_STATUS_INVALID_ARGUMENT, "tensor map: alignment/stride");
  cuuint64_t dims[3] = {(cuuint64_t)kext, (cuuint64_t)rows, (cuuint64_t)batch};
  cuuint64_t strides[2] = {(cuuint64_t)ld * 4, (cuuint64_t)ld * 4 * (cuuint64_t)rows};
  cuuint32_t box[3] = {(cuuint32_t)BK, (cuuint32_t)box_rows, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = enc(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims, strides,
                   box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(VQC_STATUS_CUDA_ERROR, "cuTensorMapEncodeTiled failed");
  return VQC_STATUS_SUCCESS;
}

template <int BN>
static int launch_half(const CUtensorMap& ta, const CUtensorMap& th, const CUtensorMap& tl,
                       const HalfParams& p, cudaStream_t st) {
  using C = HalfCfg<BN>;
  // the opt-in is a property of the current device's context: set it on every
  // launch (cheap) so a process that drives several GPUs gets it on each
  cudaError_t e = cudaFuncSetAttribute(half_ws_kernel<BN>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM);
  if (e != cudaSuccess) return cuda_status(e, "half smem attribute");
  const int grid = (p.nitems + p.per_cta - 1) / p.per_cta;
  half_ws_kernel<BN><<<grid, kHalfThreads, C::SMEM, st>>>(ta, th, tl, p);
  count_launch();
  return cuda_status(cudaGetLastError(), "half launch");
}

}  // namespace tc
}  // namespace vqc

using namespace vqc;
using namespace vqc::tc;

extern "C" int vqc_wait_selftest(int32_t budget_us, int32_t* error, void* stream) {
  if (!error || budget_us <= 0 || budget_us > 2000000)
    return fail(VQC_STATUS_INVALID_ARGUMENT, "wait_selftest: budget must be in (0, 2 s]");
  wait_selftest_kernel<<<1, 32, 0, (cudaStream_t)stream>>>(1000ull * (unsigned long long)budget_us,
                                                          error);
  count_launch();
  return cuda_status(cudaGetLastError(), "wait_selftest");
}

extern "C" int vqc_split_tf32(const float* x, float* hi, float* lo, int64_t n, void* stream) {
  if (!x || !hi || !lo || n < 0) return fail(VQC_STATUS_INVALID_ARGUMENT, "split_tf32: bad argument");
  if (n == 0) return VQC_STATUS_SUCCESS;
  long long blocks = (n + 255) / 256;
  blocks = blocks > 4096 ? 4096 : blocks;
  split_tf32_kernel<<<(int)blocks, 256, 0, (cudaStream_t)stream>>>(x, hi, lo, (size_t)n);
  count_launch();
  return cuda_status(cudaGetLastError(), "split_tf32");
}

extern "C" int vqc_tc_half_transform(const float* b_aux_major, int32_t nmol, int32_t nao,
                                     int32_t ld_ao, int32_t naux, const float* ct_hi,
                                     const float* ct_lo, const double* c_occ, int32_t nocc,
                                     int32_t o_pad, int32_t ld_aux, float* u_hi, float* u_lo,
                                     double* rho, const double* dens, double* rho_dens,
                                     int32_t* error, void* stream) {
  if (!b_aux_major || !ct_hi || !ct_lo || !c_occ || !u_hi || !u_lo || nmol <= 0 || nao <= 0 ||
      naux <= 0 || nocc <= 0 || o_pad < nocc || o_pad % 16 || o_pad > 128 || ld_ao < nao ||
      ld_aux < naux || ld_aux % 4 || (dens != nullptr) != (rho_dens != nullptr))
    return fail(VQC_STATUS_INVALID_ARGUMENT, "half_transform: bad argument");
  CUtensorMap ta, th, tl;
  int st = make_map(&ta, b_aux_major, nao, ld_ao, naux, nmol * nao, BM);
  if (!st) st = make_map(&th, ct_hi, nao, ld_ao, nocc, nmol, o_pad);
  if (!st) st = make_map(&tl, ct_lo, nao, ld_ao, nocc, nmol, o_pad);
  if (st) return st;
  HalfParams p{};
  p.nao = nao;
  p.naux = naux;
  p.nocc = nocc;
  p.ldq = ld_aux;
  p.nqt = (naux + BM - 1) / BM;
  const long long items = (long long)nmol * nao * p.nqt;
  if (items > 0x7fffffffLL) return fail(VQC_STATUS_INVALID_ARGUMENT, "half_transform: too many tiles");
  p.nitems = (int)items;
  const int ctas = p.nitems < sm_count() ? p.nitems : sm_count();
  p.per_cta = (p.nitems + ctas - 1) / ctas;
  p.nk = (nao + BK - 1) / BK;
  p.u_hi = u_hi;
  p.u_lo = u_lo;
  p.rho = rho;
  p.cvec = c_occ;
  p.dens = dens;
  p.rho_dens = rho_dens;
  p.error = error;
  cudaStream_t s = (cudaStream_t)stream;
  switch (o_pad) {
    case 16: return launch_half<16>(ta, th, tl, p, s);
    case 32: return launch_half<32>(ta, th, tl, p, s);
    case 48: return launch_half<48>(ta, th, tl, p, s);
    case 64: return launch_half<64>(ta, th, tl, p, s);
    case 80: return launch_half<80>(ta, th, tl, p, s);
    case 96: return launch_half<96>(ta, th, tl, p, s);
    case 112: return launch_half<112>(ta, th, tl, p, s);
    case 128: return launch_half<128>(ta, th, tl, p, s);
  }
  return fail(VQC_STATUS_INVALID_ARGUMENT, "half_transform: o_pad");
}

static int launch_gram(const float* a_hi, const float* a_lo, const float* b_hi, const float* b_lo,
                       int nseg, int32_t nmol, int32_t nao, int32_t kdim, double* kout,
                       int32_t* error, void* stream) {
  CUtensorMap ah, al, bh, bl;
  int st = make_map(&ah, a_hi, kdim, kdim, nao, nmol, BM);
  if (!st) st = make_map(&al, a_lo, kdim, kdim, nao, nmol, BM);
  if (!st) st = make_map(&bh, b_hi, kdim, kdim, nao, nmol, BM);
  if (!st) st = make_map(&bl, b_lo, kdim, kdim, nao, nmol, BM);
  if (st) return st;
  const int nt = (nao + BM - 1) / BM;
  const int tiles = nt * (nt + 1) / 2;
  const int kb_total = (kdim + BK - 1) / BK * nseg;
  const int sms = sm_count();
  long long base = (long long)tiles * nmol;
  // K ranges are split until about waves x SMs CTAs exist (a tuning knob)
  const long long waves = tune_value(VQC_TUNE_GRAM_WAVES);
  int ksplit = (int)((waves * sms + base - 1) / base);
  const int max_split = (kb_total + kGramFlush - 1) / kGramFlush;
  ksplit = ksplit < 1 ? 1 : (ksplit > max_split ? max_split : ksplit);
  int per = (kb_total + ksplit - 1) / ksplit;
  per = (per + kGramFlush - 1) / kGramFlush * kGramFlush;
  ksplit = (kb_total + per - 1) / per;
  if ((long long)nmol * ksplit > 65535) return fail(VQC_STATUS_INVALID_ARGUMENT, "gram: grid too large");
  GramParams p{};
  p.nao = nao;
  p.kdim = kdim;
  p.nt = nt;
  p.ntiles_ut = tiles;
  p.kblocks_per_split = per;
  p.ksplit = ksplit;
  p.nseg = nseg;
  p.kout = kout;
  p.error = error;
  // per current device (see launch_half)
  cudaError_t e = cudaFuncSetAttribute(gram_ws_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       GramCfg::SMEM);
  if (e != cudaSuccess) return cuda_status(e, "gram smem attribute");
  dim3 grid(tiles, nmol * ksplit);
  gram_ws_kernel<<<grid, kGramThreads, GramCfg::SMEM, (cudaStream_t)stream>>>(ah, al, bh, bl, p);
  count_launch();
  return cuda_status(cudaGetLastError(), "gram launch");
}

extern "C" int vqc_tc_gram(const float* u_hi, const float* u_lo, int32_t nmol, int32_t nao,
                           int32_t kdim, double* kout, int32_t* error, void* stream) {
  if (!u_hi || !u_lo || !kout || nmol <= 0 || nao <= 0 || kdim <= 0 || kdim % 4)
    return fail(VQC_STATUS_INVALID_ARGUMENT, "gram: bad argument");
  return launch_gram(u_hi, u_lo, u_hi, u_lo, 1, nmol, nao, kdim, kout, error, stream);
}

extern "C" int vqc_tc_gram_sym2(const float* a_hi, const float* a_lo, const float* b_hi,
                                const float* b_lo, int32_t nmol, int32_t nao, int32_t kdim,
                                double* kout, int32_t* error, void* stream) {
  if (!a_hi || !a_lo || !b_hi || !b_lo || !kout || nmol <= 0 || nao <= 0 || kdim <= 0 || kdim % 4)
    return fail(VQC_STATUS_INVALID_ARGUMENT, "gram_sym2: bad argument");
  return launch_gram(a_hi, a_lo, b_hi, b_lo, 2, nmol, nao, kdim, kout, error, stream);
}

extern "C" int vqc_coulomb_tma(const float* b_aux_major, const double* rho, int32_t nmol,
                               int32_t nao, int32_t ld_ao, int32_t naux, double* j, int32_t* error,
                               void* stream) {
  if (!b_aux_major || !rho || !j || !error || nmol <= 0 || nao <= 0 || naux <= 0 || ld_ao < nao ||
      ld_ao % 4 || (long long)nmol * nao > 0x7fffffffLL ||
      (naux + BM - 1) / BM * BM > kCoulMaxAux)
    return fail(VQC_STATUS_INVALID_ARGUMENT, "coulomb_tma: bad argument");
  CUtensorMap tb;
  int st = make_map(&tb, b_aux_major, nao, ld_ao, naux, nmol * nao, BM);
  if (st) return st;
  CoulParams p{};
  p.nmol = nmol;
  p.nao = nao;
  p.naux = naux;
  p.nqt = (naux + BM - 1) / BM;
  p.rho = rho;
  p.j = j;
  p.error = error;
  cudaError_t e = cudaFuncSetAttribute(coulomb_tma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       kCoulSmem);
  if (e != cudaSuccess) return cuda_status(e, "coulomb_tma smem attribute");
  const int items = nmol * nao;
  const int ctas = items < sm_count() ? items : sm_count();
  coulomb_tma_kernel<<<ctas, kCoulThreads, kCoulSmem, (cudaStream_t)stream>>>(tb, p);
  count_launch();
  return cuda_status(cudaGetLastError(), "coulomb_tma");
}
