// Split-precision (3xTF32) tensor-core GEMMs for the mixed-precision exchange.
//
// D[M x N] = A[M x K] . B[N x K]^T with FP32 operands in HBM (both K-major),
// computed on the 5th-generation tensor cores as
//     D = A_hi B_hi^T + A_hi B_lo^T + A_lo B_hi^T,
// x_hi = rn_tf32(x), x_lo = rn_tf32(x - x_hi): round-to-nearest splitting, so
// the products carry ~2^-22 relative error without the one-sided bias of
// truncation.  Operand tiles arrive by TMA (128-byte swizzle) into shared
// memory; all 128 threads split them in place (hi) and into a sibling buffer
// (lo); one thread issues tcgen05.mma (kind::tf32, M = 128) into a TMEM
// accumulator and commits to an mbarrier that releases the stage.
//
// Two epilogues:
//   kHalf  -- U = B_mu^T C (the exchange half transform, K = N_ao): FP32 store
//             of U and rho[Q] += 2 sum_i U[Q][i] C[mu][i] (the fitted density
//             that J needs), reference src/scf/cuda/df_occupied_exchange.cpp:251
//   kGram  -- K += U U^T over K = X * o (reference df_occupied_exchange.cpp:262):
//             the FP32 TMEM accumulator is drained into FP64 registers every
//             kFlush K-blocks, bounding the FP32 accumulation chain; partial
//             tiles of a split K range are added into FP64 output.
//
// Every mbarrier wait is bounded by a 2 s %globaltimer budget; on expiry the
// CTA records an error code, stops issuing work, waits (bounded) for its own
// copies and MMAs in flight, frees its TMEM and returns.
#include <cuda.h>
#include <cudaTypedefs.h>

#include "vqc_df.h"
#include "vqc_plan.hpp"

namespace vqc {
namespace tc {

constexpr int BM = 128;
constexpr int BK = 32;  // FP32 elements per K-block: one 128-byte swizzle row
constexpr int THREADS = 128;
constexpr int kFlush = 4;  // K-blocks per FP32 accumulation chain in kGram
constexpr unsigned long long kWaitNs = 2000000000ull;

enum Mode { kHalf = 0, kGram = 1 };

struct Params {
  int m, n, kdim;
  int kblocks_per_split, ksplit;
  int b_batch_div;
  float* u;          // kHalf: [z][m][ldu]
  int ldu;
  double* rho;       // kHalf: [z / rho_div][m]
  const double* cvec;  // kHalf: [z][cld]
  int cld, ncvec, rho_div;
  double* kout;      // kGram: [z][m][n]
  int* error;
};

template <int BN>
struct Cfg {
  static constexpr int A_BYTES = BM * BK * 4;
  static constexpr int B_BYTES = BN * BK * 4;
  static constexpr int STAGE = 2 * A_BYTES + 2 * B_BYTES;
  static constexpr int STAGES = (220 * 1024) / STAGE >= 4 ? 4 : (220 * 1024) / STAGE;
  static constexpr int SMEM = STAGES * STAGE + 1024 + 256;
  static constexpr int TMEM_COLS = BN <= 32 ? 32 : (BN <= 64 ? 64 : (BN <= 128 ? 128 : 256));
  static_assert(BN % 16 == 0 && BN >= 16 && BN <= 256, "M=128 tf32 MMA needs N % 16 == 0");
  static_assert(STAGES >= 2, "shared memory too small for the pipeline");
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}

// bounded wait; false on timeout or when *abort is set
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort) {
  const unsigned long long t0 = globaltimer();
  while (true) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    if (ok) return true;
    if (*abort) return false;
    if (globaltimer() - t0 > kWaitNs) return false;
  }
}

__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* tm, int c0, int c1,
                                            int c2, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(tm)), "r"(c0), "r"(c1), "r"(c2), "r"(bar)
      : "memory");
}

// K-major, 128-byte swizzle, 8-row groups 1024 bytes apart (SBO), version 1
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
  return (uint64_t)((addr & 0x3FFFFu) >> 4) | (1ull << 16) | (64ull << 32) | (1ull << 46) |
         (2ull << 61);
}

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

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   bar)
               : "memory");
}

__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
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

__device__ __forceinline__ float rn_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

__device__ __forceinline__ void split4(float4& v, float4& lo) {
  float h;
  h = rn_tf32(v.x); lo.x = rn_tf32(v.x - h); v.x = h;
  h = rn_tf32(v.y); lo.y = rn_tf32(v.y - h); v.y = h;
  h = rn_tf32(v.z); lo.z = rn_tf32(v.z - h); v.z = h;
  h = rn_tf32(v.w); lo.w = rn_tf32(v.w - h); v.w = h;
}

template <int BN, int MODE>
__global__ void __launch_bounds__(THREADS, 1)
    tf32x3_gemm_kernel(const __grid_constant__ CUtensorMap tmA,
                       const __grid_constant__ CUtensorMap tmB, Params p) {
  using C = Cfg<BN>;
  constexpr int S = C::STAGES;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + S * C::STAGE);
  // bars[0..S): full, bars[S..2S): empty, bars[2S]: accumulator ready
  volatile uint32_t* tmem_slot = reinterpret_cast<volatile uint32_t*>(bars + 2 * S + 1);
  volatile int* abort = reinterpret_cast<volatile int*>(bars + 2 * S + 2);

  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const int z = blockIdx.z / p.ksplit, split = blockIdx.z % p.ksplit;
  const int zb = z / p.b_batch_div;
  const int row0 = blockIdx.x * BM, col0 = blockIdx.y * BN;
  const int kb_total = (p.kdim + BK - 1) / BK;
  const int kb0 = split * p.kblocks_per_split;
  const int kb1 = min(kb_total, kb0 + p.kblocks_per_split);
  const int nkb = kb1 - kb0;
  if (nkb <= 0) return;  // uniform per CTA

  const uint32_t full0 = smem_u32(bars), empty0 = smem_u32(bars + S), accb = smem_u32(bars + 2 * S);
  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(full0 + 8 * s, 1);
      mbar_init(empty0 + 8 * s, 1);
    }
    mbar_init(accb, 1);
    *abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(const_cast<uint32_t*>(tmem_slot))),
                 "r"(C::TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = *tmem_slot;
  constexpr uint32_t idesc = instr_desc<BN>();
  constexpr uint32_t TX = C::A_BYTES + C::B_BYTES;

  auto stage_ptr = [&](int s) { return smem + s * C::STAGE; };
  // producer prologue
  int issued = 0;
  if (tid == 0) {
    for (; issued < S && issued < nkb; ++issued) {
      const int s = issued;
      const uint32_t a = smem_u32(stage_ptr(s));
      mbar_expect_tx(full0 + 8 * s, TX);
      tma_load_3d(a, &tmA, (kb0 + issued) * BK, row0, z, full0 + 8 * s);
      tma_load_3d(a + 2 * C::A_BYTES, &tmB, (kb0 + issued) * BK, col0, zb, full0 + 8 * s);
    }
  }

  double acc64[MODE == kGram ? BN : 1];
#pragma unroll
  for (int c = 0; c < (MODE == kGram ? BN : 1); ++c) acc64[c] = 0.0;
  int flushes = 0;
  bool chain_start = true;
  int mma_commits = 0;

  int consumed = 0;  // k-blocks whose full barrier every thread has passed
  for (int i = 0; i < nkb; ++i) {
    const int s = i % S;
    const uint32_t ph = (i / S) & 1;
    const bool ok = mbar_wait(full0 + 8 * s, ph, abort);
    if (!ok) {
      if (p.error) atomicExch(p.error, 1);
      *abort = 1;
    } else {
      // split the tile: hi in place, lo into the sibling buffer
      float4* a = reinterpret_cast<float4*>(stage_ptr(s));
      float4* alo = reinterpret_cast<float4*>(stage_ptr(s) + C::A_BYTES);
      float4* b = reinterpret_cast<float4*>(stage_ptr(s) + 2 * C::A_BYTES);
      float4* blo = reinterpret_cast<float4*>(stage_ptr(s) + 2 * C::A_BYTES + C::B_BYTES);
#pragma unroll 4
      for (int k = tid; k < C::A_BYTES / 16; k += THREADS) {
        float4 v = a[k], lo;
        split4(v, lo);
        a[k] = v;
        alo[k] = lo;
      }
#pragma unroll 4
      for (int k = tid; k < C::B_BYTES / 16; k += THREADS) {
        float4 v = b[k], lo;
        split4(v, lo);
        b[k] = v;
        blo[k] = lo;
      }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    fence_before_sync();
    __syncthreads();
    if (*abort) break;  // uniform: read after the barrier
    consumed = i + 1;
    if (tid == 0) {
      fence_after_sync();
      const uint32_t ahi = smem_u32(stage_ptr(s)), alo = ahi + C::A_BYTES;
      const uint32_t bhi = ahi + 2 * C::A_BYTES, blo = bhi + C::B_BYTES;
#pragma unroll
      for (int kk = 0; kk < BK / 8; ++kk) {
        const uint32_t off = kk * 32;  // 8 tf32 = 32 bytes along K
        mma_tf32(tmem, smem_desc(alo + off), smem_desc(bhi + off), idesc,
                 (chain_start && kk == 0) ? 0u : 1u);
        mma_tf32(tmem, smem_desc(ahi + off), smem_desc(blo + off), idesc, 1u);
        mma_tf32(tmem, smem_desc(ahi + off), smem_desc(bhi + off), idesc, 1u);
      }
      mma_commit(empty0 + 8 * s);
      ++mma_commits;
      // refill the stage the previous k-block used
      if (i >= 1) {
        const int j = i - 1 + S;
        const int sp = (i - 1) % S;
        if (j < nkb) {
          if (!mbar_wait(empty0 + 8 * sp, ((i - 1) / S) & 1, abort)) {
            if (p.error) atomicExch(p.error, 2);
            *abort = 1;
          } else {
            const uint32_t a = smem_u32(stage_ptr(sp));
            mbar_expect_tx(full0 + 8 * sp, TX);
            tma_load_3d(a, &tmA, (kb0 + j) * BK, row0, z, full0 + 8 * sp);
            tma_load_3d(a + 2 * C::A_BYTES, &tmB, (kb0 + j) * BK, col0, zb, full0 + 8 * sp);
            ++issued;
          }
        }
      }
    }
    chain_start = false;
    const bool last = (i == nkb - 1);
    if (MODE == kGram && ((i + 1) % kFlush == 0 || last)) {
      if (tid == 0) mma_commit(accb);
      if (!mbar_wait(accb, flushes & 1, abort)) {
        if (p.error) atomicExch(p.error, 3);
        *abort = 1;
      }
      __syncthreads();
      if (*abort) break;  // uniform
      ++flushes;
      fence_after_sync();
#pragma unroll
      for (int c = 0; c < BN; c += 16) {
        float v[16];
        tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + c, v);
#pragma unroll
        for (int q = 0; q < 16; ++q) acc64[c + q] += (double)v[q];
      }
      fence_before_sync();
      __syncthreads();
      chain_start = true;
    }
  }
  // the barrier-read flag is uniform from here on
  __syncthreads();

  if (!*abort && MODE == kHalf) {
    if (tid == 0) mma_commit(accb);
    if (!mbar_wait(accb, 0, abort)) {
      if (p.error) atomicExch(p.error, 4);
      *abort = 1;
    }
    __syncthreads();
    if (!*abort) {
      fence_after_sync();
      const int row = row0 + tid;
      double rho_part = 0.0;
#pragma unroll
      for (int c = 0; c < BN; c += 16) {
        float v[16];
        tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + c, v);
        if (row < p.m) {
          float* dst = p.u + ((size_t)z * p.m + row) * p.ldu;
#pragma unroll
          for (int q = 0; q < 16; ++q) {
            const int col = col0 + c + q;
            if (col < p.ldu) dst[col] = v[q];
            if (col < p.ncvec) rho_part += (double)v[q] * p.cvec[(size_t)z * p.cld + col];
          }
        }
      }
      if (row < p.m && p.rho) atomicAdd(p.rho + (size_t)(z / p.rho_div) * p.m + row, 2.0 * rho_part);
    }
  }
  if (!*abort && MODE == kGram) {
    const int row = row0 + tid;
    if (row < p.m) {
      double* dst = p.kout + ((size_t)z * p.m + row) * p.n;
#pragma unroll
      for (int c = 0; c < BN; ++c) {
        const int col = col0 + c;
        if (col < p.n) atomicAdd(dst + col, acc64[c]);
      }
    }
  }

  if (*abort && tid == 0) {
    // drain: copies still in flight land in this CTA's shared memory and the
    // last committed MMAs still read it and write TMEM; wait for both (bounded)
    volatile int never = 0;
    for (int i2 = consumed; i2 < issued; ++i2)
      mbar_wait(full0 + 8 * (i2 % S), (i2 / S) & 1, &never);
    if (mma_commits > 0) {
      const int lastc = mma_commits - 1;
      mbar_wait(empty0 + 8 * (lastc % S), (lastc / S) & 1, &never);
    }
  }
  fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    fence_after_sync();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(C::TMEM_COLS)
                 : "memory");
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    cudaDriverEntryPointQueryResult q;
    void* f = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  }
  return fn;
}

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

template <int BN, int MODE>
static int launch(const CUtensorMap& ta, const CUtensorMap& tb, const Params& p, dim3 grid,
                  cudaStream_t st) {
  using C = Cfg<BN>;
  auto k = tf32x3_gemm_kernel<BN, MODE>;
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM);
    if (e != cudaSuccess) return cuda_status(e, "tf32x3 smem attribute");
    attr = true;
  }
  k<<<grid, THREADS, C::SMEM, st>>>(ta, tb, p);
  count_launch();
  return cuda_status(cudaGetLastError(), "tf32x3 launch");
}

}  // namespace tc
}  // namespace vqc

using namespace vqc;
using namespace vqc::tc;

extern "C" int vqc_tc_half_transform(const float* b_aux_major, int32_t nmol, int32_t nao,
                                     int32_t ld_ao, int32_t naux, const float* ct,
                                     const double* c_occ, int32_t nocc, int32_t o_pad, float* u,
                                     double* rho, int32_t* error, void* stream) {
  if (!b_aux_major || !ct || !c_occ || !u || nmol <= 0 || nao <= 0 || naux <= 0 || nocc <= 0 ||
      o_pad < nocc || o_pad % 16 || o_pad > 128 || ld_ao < nao)
    return fail(VQC_STATUS_INVALID_ARGUMENT, "half_transform: bad argument");
  CUtensorMap ta, tb;
  int st = make_map(&ta, b_aux_major, nao, ld_ao, naux, nmol * nao, BM);
  if (!st) st = make_map(&tb, ct, nao, ld_ao, nocc, nmol, o_pad);
  if (st) return st;
  Params p{};
  p.m = naux;
  p.n = o_pad;
  p.kdim = nao;
  p.kblocks_per_split = (nao + BK - 1) / BK;
  p.ksplit = 1;
  p.b_batch_div = nao;
  p.u = u;
  p.ldu = o_pad;
  p.rho = rho;
  p.cvec = c_occ;
  p.cld = nocc;
  p.ncvec = nocc;
  p.rho_div = nao;
  p.error = error;
  if ((long long)nmol * nao > 65535) return fail(VQC_STATUS_INVALID_ARGUMENT, "half_transform: grid too large");
  dim3 grid((naux + BM - 1) / BM, 1, nmol * nao);
  cudaStream_t s = (cudaStream_t)stream;
  switch (o_pad) {
    case 16: return launch<16, kHalf>(ta, tb, p, grid, s);
    case 32: return launch<32, kHalf>(ta, tb, p, grid, s);
    case 48: return launch<48, kHalf>(ta, tb, p, grid, s);
    case 64: return launch<64, kHalf>(ta, tb, p, grid, s);
    case 80: return launch<80, kHalf>(ta, tb, p, grid, s);
    case 96: return launch<96, kHalf>(ta, tb, p, grid, s);
    case 112: return launch<112, kHalf>(ta, tb, p, grid, s);
    case 128: return launch<128, kHalf>(ta, tb, p, grid, s);
  }
  return fail(VQC_STATUS_INVALID_ARGUMENT, "half_transform: o_pad");
}

extern "C" int vqc_tc_gram(const float* u, int32_t nmol, int32_t nao, int32_t kdim, double* kout,
                           int32_t* error, void* stream) {
  if (!u || !kout || nmol <= 0 || nao <= 0 || kdim <= 0 || kdim % 4)
    return fail(VQC_STATUS_INVALID_ARGUMENT, "gram: bad argument");
  constexpr int BN = 64;
  CUtensorMap ta, tb;
  int st = make_map(&ta, u, kdim, kdim, nao, nmol, BM);
  if (!st) st = make_map(&tb, u, kdim, kdim, nao, nmol, BN);
  if (st) return st;
  const int mt = (nao + BM - 1) / BM, nt = (nao + BN - 1) / BN;
  const int kb_total = (kdim + BK - 1) / BK;
  int sms = 148;
  int dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long tiles = (long long)mt * nt * nmol;
  int ksplit = (int)((2LL * sms + tiles - 1) / tiles);
  ksplit = ksplit < 1 ? 1 : ksplit;
  const int max_split = (kb_total + kFlush - 1) / kFlush;
  ksplit = ksplit > max_split ? max_split : ksplit;
  int per = (kb_total + ksplit - 1) / ksplit;
  per = (per + kFlush - 1) / kFlush * kFlush;
  ksplit = (kb_total + per - 1) / per;
  Params p{};
  p.m = nao;
  p.n = nao;
  p.kdim = kdim;
  p.kblocks_per_split = per;
  p.ksplit = ksplit;
  p.b_batch_div = 1;
  p.kout = kout;
  p.error = error;
  if ((long long)nmol * ksplit > 65535) return fail(VQC_STATUS_INVALID_ARGUMENT, "gram: grid too large");
  dim3 grid(mt, nt, nmol * ksplit);
  return launch<BN, kGram>(ta, tb, p, grid, (cudaStream_t)stream);
}
