/*
 * vqc_df.h -- C ABI of the B200 DF-RHF engine (libvqc_b200.so).
 *
 * Plain C: device pointers, host pointers, sizes and a cudaStream_t passed as
 * void*. No C++ or torch types cross this boundary.  Every entry point returns
 * a status in the reference's generativeqc_status vocabulary
 * (include/generativeqc/generativeqc.h:23-42 of the reference):
 *   0 success, 1 invalid argument, 2 ABI mismatch (a descriptor whose
 *   struct_size/abi_version this library does not accept), 4 not converged,
 *   5 numerical failure, 6 CUDA error, 7 out of memory.
 * A thread-local detail string is available from vqc_last_error() (same idea as
 * generativeqc_context_get_last_detail, generativeqc.h:1231).
 *
 * Ownership: the caller owns every input and output buffer; the library
 * allocates only inside a vqc_plan (device copies of the batch topology), which
 * vqc_plan_destroy releases (docs/developer/architecture.md:149-153 of the
 * reference: caller-provided output storage remains caller-owned).
 * Threading: a plan is not re-entrant; callers serialise use of one plan.
 */
#ifndef VQC_DF_H
#define VQC_DF_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VQC_ABI_VERSION 1u

enum {
  VQC_STATUS_SUCCESS = 0,
  VQC_STATUS_INVALID_ARGUMENT = 1,
  VQC_STATUS_ABI_MISMATCH = 2,
  VQC_STATUS_NOT_CONVERGED = 4,
  VQC_STATUS_NUMERICAL_FAILURE = 5,
  VQC_STATUS_CUDA_ERROR = 6,
  VQC_STATUS_OUT_OF_MEMORY = 7
};

typedef struct vqc_plan vqc_plan;

/*
 * A ragged batch of molecules with their orbital and auxiliary shells (host
 * arrays).  Replaces the per-system generativeqc_system_descriptor
 * (generativeqc.h:586-599: atoms, shells, primitives) plus the auxiliary-basis
 * system handle (generativeqc.h:733-740), batched the way
 * generativeqc_batch_prepare (generativeqc.h:1435) receives a list of systems.
 * Shell atom indices are global (into the concatenated atom list).  Primitive
 * coefficients already include primitive and contraction normalisation.
 * Auxiliary shells must be sorted by angular momentum within each molecule.
 */
typedef struct {
  uint32_t struct_size;
  uint32_t abi_version;
  int32_t nmol;
  int32_t spherical;                 /* 1: real spherical, 0: Cartesian */
  const int32_t* mol_atom_offset;    /* [nmol+1] */
  const int32_t* mol_shell_offset;   /* [nmol+1] orbital shells */
  const int32_t* mol_aux_offset;     /* [nmol+1] auxiliary shells */
  const double* atom_charge;         /* [natom] nuclear charges */
  const int32_t* shell_l;            /* orbital shells */
  const int32_t* shell_atom;
  const int32_t* shell_nprim;
  const int32_t* shell_prim_off;
  const double* prim_exp;
  const double* prim_coef;
  int32_t nprim;
  const int32_t* aux_l;              /* auxiliary shells */
  const int32_t* aux_atom;
  const int32_t* aux_nprim;
  const int32_t* aux_prim_off;
  const double* aux_exp;
  const double* aux_coef;
  int32_t naux_prim;
} vqc_batch_desc;

/* Per-molecule sizes and offsets (elements) into the batch-wide buffers. */
typedef struct {
  int32_t nao;        /* orbital functions N */
  int32_t naux;       /* auxiliary functions X */
  int32_t natom;
  int32_t atom_offset;
  int64_t mat_offset; /* into N*N buffers (S, T, V, D, J, K, F) */
  int64_t met_offset; /* into X*X buffers (metric) */
  int64_t a_offset;   /* into packed 3-centre buffers: N(N+1)/2 rows of X */
} vqc_molecule_info;

const char* vqc_last_error(void);
uint32_t vqc_abi_version(void);
/* Number of kernel launches this library has issued (process lifetime). */
uint64_t vqc_launch_count(void);

/*
 * Tuning knobs read by the kernels' launchers (process-wide; set between
 * launches, e.g. from an autotuned table per batch shape).  No counterpart
 * in the reference, whose CUDA schedules come from build-time tuning
 * manifests (python/generativeqc_compiler/integral/df_tuning/).
 *   VQC_TUNE_GRAM_WAVES: the exchange Gram product splits its K range until
 *     about this many CTAs per SM exist (1..64, default 2).
 */
enum { VQC_TUNE_GRAM_WAVES = 1, VQC_TUNE_COUNT = 2 };
int vqc_tune_set(int32_t knob, int32_t value);
int vqc_tune_get(int32_t knob, int32_t* value);

/* Plan over a batch topology (generativeqc_batch_prepare, generativeqc.h:1435). */
int vqc_plan_create(const vqc_batch_desc* desc, vqc_plan** out);
int vqc_plan_destroy(vqc_plan* plan);
int vqc_plan_totals(const vqc_plan* plan, int64_t* mat_total, int64_t* met_total,
                    int64_t* a_total, int32_t* natom_total);
int vqc_plan_molecule(const vqc_plan* plan, int32_t index, vqc_molecule_info* info);

/*
 * Integrals.  xyz: device [natom][3] Bohr.  Outputs are device buffers sized
 * by vqc_plan_totals.
 *   vqc_int1e  -> S, T, V (each mat_total)      reference s_integrals.cpp:1865
 *   vqc_int2c  -> metric (P|Q) (met_total)      reference s_integrals.cpp:1201
 *   vqc_int3c  -> A[(mu nu) packed, mu>=nu][P]  reference s_integrals.cpp:1201,
 *                 df_source_kernels.cu:67 (raw tiles, aux contiguous)
 */
int vqc_int1e(vqc_plan* plan, const double* xyz, double* s, double* t, double* v, void* stream);
int vqc_int2c(vqc_plan* plan, const double* xyz, double* metric, void* stream);
int vqc_int3c(vqc_plan* plan, const double* xyz, double* a_packed, void* stream);
/* Bounded 3-centre row tiles: the packed rows of one molecule whose larger AO
 * index mu lies in the functions of its orbital shells [shell_begin,
 * shell_end) (shell indices counted within the molecule), i.e. rows
 * mu(mu+1)/2 + nu - f0(f0+1)/2 for f0 <= mu < f1, nu <= mu, where f0 / f1 are
 * the first functions of shell_begin / shell_end: (f1(f1+1)/2 - f0(f0+1)/2) x
 * naux doubles, the same values vqc_int3c writes there.  Replaces the
 * reference's bounded DF integral source tiles
 * (src/scf/cuda/df_source.cpp:347-372, generate_cuda_density_fitting_raw_tile)
 * for recompute under a memory bound.  Calls on one plan are stream-ordered:
 * they share a small work table inside the plan. */
int vqc_int3c_rows(vqc_plan* plan, const double* xyz, int32_t mol, int32_t shell_begin,
                   int32_t shell_end, double* rows, void* stream);

/*
 * Gradient contractions (accumulate into grad[natom][3]; the caller zeroes it).
 *   vqc_grad3c: g += sum Abar[(mu nu) packed][P] d(mu nu|P)/dR, with Abar
 *               symmetric in (mu, nu) and stored like vqc_int3c's output.
 *               Replaces generativeqc_system_df_gradient_cuda's 3-centre part
 *               (generativeqc.h:1312-1333; src/api/c_api_df_gradient.cpp:11).
 *   vqc_grad2c: g += sum Mbar[P][Q] d(P|Q)/dR (same entry's metric part).
 *   vqc_grad1e: g += sum D d(T+V)/dR - W dS/dR, nuclear-position terms included
 *               (reference src/integrals/s_integrals.cpp:2187).
 */
int vqc_grad3c(vqc_plan* plan, const double* xyz, const double* abar_packed, double* grad,
               void* stream);
int vqc_grad2c(vqc_plan* plan, const double* xyz, const double* mbar, double* grad, void* stream);
int vqc_grad1e(vqc_plan* plan, const double* xyz, const double* dens, const double* wdens,
               double* grad, void* stream);

/*
 * Standalone DF gradient contraction with the contract of the reference's
 * generativeqc_system_df_gradient_cuda (include/generativeqc/generativeqc.h:
 * 1312-1333; src/api/c_api_df_gradient.cpp:11):
 *   gradient[a][x] = sum_{mu,nu,P} bar_a[mu][nu][P] d(mu nu|P)/dR_ax
 *                  + sum_{P,Q} bar_m[P][Q] d(P|Q)/dR_ax
 * system: exactly one molecule (its orbital and auxiliary shells); xyz: HOST
 * [natom][3] Bohr.  bar_a: HOST full row-major [mu][nu][P], count_a = N*N*X;
 * bar_m: HOST full row-major [P][Q], count_m = X*X; either may be NULL
 * (that channel is zero; the counts must still match).  Nonsymmetric weights
 * are allowed and every element is counted once.  gradient: HOST [natom][3],
 * gradient_count = 3*natom, DF terms only; written only on success (failures
 * leave it untouched).  maximum_bytes (> 0) bounds the device memory of the
 * weights: bar_a is streamed in auxiliary-shell column tiles of at most
 * maximum_tile_elements (0: automatic) elements of N*N*X_tile.
 * schedule 0 or 1 (the reference's thread / serial traversal) selects the
 * same kernels here; their floating-point atomics make the summation order,
 * hence the last bits, vary between calls.  resources (optional; struct_size
 * and abi_version must be set, else status 2) receives the staging record.
 * Runs on the current device's default stream and synchronises before it
 * returns.
 */
typedef struct {
  uint32_t struct_size;
  uint32_t abi_version;
  uint64_t host_bytes, device_bytes, host_to_device_bytes, device_to_host_bytes;
  uint64_t weight_tile_elements, tiles, uploads, stream_synchronizations;
} vqc_df_gradient_resources;

int vqc_df_gradient(const vqc_batch_desc* system, const double* xyz, const double* bar_a,
                    size_t count_a, const double* bar_m, size_t count_m, uint32_t schedule,
                    size_t maximum_bytes, size_t maximum_tile_elements, double* gradient,
                    size_t gradient_count, vqc_df_gradient_resources* resources);

/*
 * FP64-accurate products on the int8 tensor cores (slices of 7 bits with exact
 * int32 accumulation; tcgen05.mma kind::i8).  Used for the whitening
 * B = A W of the mixed-precision path (reference src/scf/density_fitting.cpp:
 * 711-764 and src/scf/cuda/df_plan_setup.cpp:34,70, an FP64 GEMM there).
 *   vqc_ozaki_slice_rows: rows of src (nmol blocks of `rows` rows, row stride
 *     ld, block stride mol_stride; each element times col_scale[mol][col]
 *     when col_scale is not NULL -- exact powers of two) -> exps[mol][row]
 *     (max |row| < 2^e) and nslices (1..7) int8 slices
 *     dst[mol][slice][row][ldd] with row * 2^-e = sum_s dst_s 2^-7s + r,
 *     |r| <= 2^-7 nslices.  Columns >= cols of dst are not written.
 *   vqc_ozaki_gemm: c[mol][r][n] (row stride ldc, block stride c_mol_stride)
 *     = sum_k A[mol][r][k] B[mol][n][k] from the slices of A (m rows) and B
 *     (n rows), both [mol][slice][row][ldk] (ldk % 16 == 0, k <= ldk) with
 *     their exponents, keeping slice pairs s + t <= nslices + 1.  upper = 1:
 *     B[mol][n][k] = 0 for k > n (only those K are read); upper = 2: A and B
 *     are the same slices (m == n) and C is symmetric: only the tiles on or
 *     above the diagonal are formed and each element above the diagonal is
 *     also written to its mirror (the sliced sums are exactly symmetric).
 *     k * nslices *
 *     127^2 must stay below 2^31.  error: device int set non-zero when a
 *     bounded wait expires (the output is then invalid).
 */
int vqc_ozaki_slice_rows(const double* src, int32_t nmol, int64_t rows, int32_t cols, int64_t ld,
                         int64_t mol_stride, const double* col_scale, int32_t nslices, int8_t* dst,
                         int32_t ldd, int32_t* exps, void* stream);
int vqc_ozaki_gemm(const int8_t* a_slices, const int32_t* a_exps, int64_t m, const int8_t* b_slices,
                   const int32_t* b_exps, int32_t n, int32_t k, int32_t ldk, int32_t nmol,
                   int32_t nslices, int32_t upper, double* c, int64_t ldc, int64_t c_mol_stride,
                   int32_t* error, void* stream);

/*
 * One SP2 purification step for nmol molecules of one size n (row-major n*n
 * blocks, contiguous): xout = x2 or 2x - x2 per molecule (x2 = x x), chosen to
 * move tr x toward nocc; molecules with |tr x - tr x2| < tol are copied and
 * flagged in done[nmol].  Replaces the batched Fock eigensolve of the
 * reference's device SCF loop (src/scf/cuda/df_scf_library.cpp) for the
 * density update.
 */
int vqc_sp2_update(const double* x, const double* x2, double* xout, int32_t nmol, int32_t n,
                   double nocc, double tol, int32_t* done, void* stream);

/*
 * Mixed-precision J/K over the FP32 whitened tensor stored aux-major per AO
 * row: b_aux_major[mol][mu][Q][nu], row length ld_ao >= nao (ld_ao % 4 == 0;
 * the Coulomb and fitted-density kernels take ld_ao <= 512,
 * padding zero).  Replaces the FP64 packed/dense B of the reference's CUDA
 * plan (src/scf/cuda/df_plan_setup.cpp:70,224).
 *   vqc_unpack_aux_major: packed whitened FP64 rows -> b_aux_major (FP32).
 *   vqc_split_tf32: hi = rn_tf32(x), lo = rn_tf32(x - hi) (n FP32 values).
 *   vqc_tc_half_transform: U[mol][mu][i][Q] = sum_nu B[mu][Q][nu] C[nu][i]
 *     (3xTF32 tcgen05; i < nocc, Q rows of length ld_aux >= naux, ld_aux % 4
 *     == 0, padding left untouched), written split as u_hi/u_lo (FP32,
 *     TF32-representable), and rho[mol][Q] += 2 sum_{mu,i} U C[mu][i];
 *     ct_hi/ct_lo = split C^T [mol][nocc][ld_ao] FP32, c_occ = C
 *     [mol][nao][nocc] FP64; o_pad = MMA N (round_up(nocc,16) <= 128).
 *     With dens (D [mol][nao][nao] FP64, NULL to skip) the same pass also
 *     adds the fitted density rho_dens[mol][Q] += sum_{mu,nu} B[mu][Q][nu]
 *     D[mu][nu] (four-term FP32 partial sums of the exact FP32 B values
 *     times D rounded to FP32, accumulated in FP64: error within a few 2^-24
 *     of sum |B| |D|; dens and rho_dens both set or both NULL), so a build
 *     needs no separate fitted-density pass over B.
 *     Reference src/scf/cuda/df_occupied_exchange.cpp:251-257 (U = B C) and
 *     src/scf/cuda/df_coulomb.cpp:38-57 (rho = B^T vec(D)).
 *   vqc_tc_gram: kout[mol] += U U^T over kdim = nocc * ld_aux from the split
 *     U (3xTF32, FP64 output); reference df_occupied_exchange.cpp:262-279.
 *   vqc_tc_gram_sym2: kout[mol] += A B^T + B A^T for two split operands of
 *     the same layout; forms the incremental exchange about an FP64 anchor,
 *     K(D) = K(D0) + 2 (V dU^T + dU V^T) with dU = B (C - C0) and
 *     V = U0 + dU / 2 (no counterpart in the reference, which rebuilds K in
 *     FP64 every iteration).
 *   vqc_coulomb_fp32: J[mol][mu][nu] = sum_Q B[mu][Q][nu] rho[mol][Q] (FP64
 *     accumulate); reference src/scf/cuda/df_coulomb.cpp:24.
 *   vqc_fitted_density_fp32: rho[mol][Q] = sum_{mu,nu} B[mu][Q][nu] D[mu][nu]
 *     for symmetric D [mol][nao][nao] (FP64 accumulate, deterministic);
 *     partial: caller-owned workspace of nmol * nao * naux doubles (the
 *     per-AO-row partial sums); reference df_coulomb.cpp:38-57.
 *   vqc_anchor_combine: with the FP64 anchor u0[rows][x] and the split
 *     increment du_hi/du_lo[rows][ld_aux]: mode 0 writes the split
 *     V = u0 + alpha (du_hi + du_lo) into v_hi/v_lo[rows][ld_aux] (padding
 *     zero); mode 1 adds alpha (du_hi + du_lo) into u0 in place.  No
 *     counterpart in the reference.
 * error: device int set non-zero when a bounded wait inside a tensor-core
 * kernel expires (the kernel then stops early; the caller must treat the
 * output as invalid).
 */
int vqc_unpack_aux_major(const double* b_packed, int32_t nmol, int32_t nao, int32_t naux,
                         int32_t ld_ao, float* b_aux_major, void* stream);
int vqc_split_tf32(const float* x, float* hi, float* lo, int64_t n, void* stream);
/* Self-test of the tensor-core kernels' bounded waits: a one-warp kernel waits
 * on a barrier that nothing completes, gives up after budget_us microseconds
 * (<= 2 s) and writes 31 to *error; the context stays usable.  No counterpart
 * in the reference. */
int vqc_wait_selftest(int32_t budget_us, int32_t* error, void* stream);
int vqc_tc_half_transform(const float* b_aux_major, int32_t nmol, int32_t nao, int32_t ld_ao,
                          int32_t naux, const float* ct_hi, const float* ct_lo,
                          const double* c_occ, int32_t nocc, int32_t o_pad, int32_t ld_aux,
                          float* u_hi, float* u_lo, double* rho, const double* dens,
                          double* rho_dens, int32_t* error, void* stream);
int vqc_tc_gram(const float* u_hi, const float* u_lo, int32_t nmol, int32_t nao, int32_t kdim,
                double* kout, int32_t* error, void* stream);
int vqc_tc_gram_sym2(const float* a_hi, const float* a_lo, const float* b_hi, const float* b_lo,
                     int32_t nmol, int32_t nao, int32_t kdim, double* kout, int32_t* error,
                     void* stream);
/*
 * vqc_fitted_density_fp32_noalloc: vqc_fitted_density_fp32 for callers that
 * cannot allocate device memory (their GPU memory belongs to another
 * allocator's pool, or they must avoid the synchronisation cudaFree implies).
 * The caller passes only inputs and the output; the partial sums use a fixed
 * device array of 4194304 doubles (32 MiB) inside the library, held on every
 * GPU that loads it until exit, so nmol * nao * naux must not exceed 4194304
 * (larger requests fail with VQC_STATUS_INVALID_ARGUMENT).  Allocates nothing.
 * The first call on a device looks up the array's address (make it before
 * any stream capture).  The array keeps the last call's contents and nothing
 * in it needs zeroing.  Calls that overlap on the GPU share the array and
 * race: serialise them.  No counterpart in the reference.
 */
int vqc_fitted_density_fp32_noalloc(const float* b_aux_major, const double* dens, int32_t nmol,
                                    int32_t nao, int32_t ld_ao, int32_t naux, double* rho,
                                    void* stream);
int vqc_anchor_combine(double* u0, const float* du_hi, const float* du_lo, float* v_hi,
                       float* v_lo, int64_t rows, int32_t x, int32_t ld_aux, double alpha,
                       int32_t mode, void* stream);
/* vqc_coulomb_tma: the Coulomb build of vqc_coulomb_fp32 streamed by TMA
 * (persistent CTAs, a ring of 16 KB stages, FP64 accumulation; no limit on
 * ld_ao); error: device int set non-zero when a bounded wait expires (the
 * output is then invalid).  Reference src/scf/cuda/df_coulomb.cpp:24. */
int vqc_coulomb_tma(const float* b_aux_major, const double* rho, int32_t nmol, int32_t nao,
                    int32_t ld_ao, int32_t naux, double* j, int32_t* error, void* stream);
int vqc_coulomb_fp32(const float* b_aux_major, const double* rho, int32_t nmol, int32_t nao,
                     int32_t ld_ao, int32_t naux, double* j, void* stream);
int vqc_fitted_density_fp32(const float* b_aux_major, const double* dens, int32_t nmol,
                            int32_t nao, int32_t ld_ao, int32_t naux, double* partial, double* rho,
                            void* stream);

#ifdef __cplusplus
}
#endif

#endif /* VQC_DF_H */
