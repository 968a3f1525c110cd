// Standalone DF gradient contraction with the contract of the reference's
// generativeqc_system_df_gradient_cuda (include/generativeqc/generativeqc.h:
// 1312-1333; src/api/c_api_df_gradient.cpp:11): fixed external weights
// bar_a[mu][nu][P] and bar_m[P][Q] (full row-major host arrays, nonsymmetric
// allowed, every element counted once) contracted with the derivative 3- and
// 2-centre integrals of one molecule; output [atom][xyz] on the host, written
// only on success.
//
// The derivative integrals are symmetric in (mu, nu) and in (P, Q), so the
// contraction only sees the symmetric parts of the weights:
//   sum_{mu nu P} bar_a d(mu nu|P) = sum_{mu >= nu} sym(bar_a)[mu nu][P] ...
// with the ordered-pair counting of the plan's grad3c/grad2c kernels.  bar_a
// is streamed in column tiles (aligned to auxiliary shells) under the caller's
// memory bound: each tile is copied as N*N rows of the tile width, packed and
// symmetrised on the device, and contracted by the grad3c kernels through a
// tile view of the molecule (row stride = tile width, column origin = tile
// start).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <memory>
#include <string>
#include <vector>

#include "vqc_df.h"
#include "vqc_kernels.cuh"
#include "vqc_plan.hpp"

namespace vqc {
namespace {

// packed[r][c] = (full[mu][nu][c] + full[nu][mu][c]) / 2, r = mu (mu+1)/2 + nu,
// nu <= mu, for a tile of width w (rows of the full tile are contiguous)
__global__ void pack_symmetric_tile_kernel(const double* __restrict__ full, int n, int w,
                                           double* __restrict__ packed) {
  const long long rows = (long long)n * (n + 1) / 2;
  for (long long r = blockIdx.x; r < rows; r += gridDim.x) {
    long long mu = (long long)((sqrt(8.0 * (double)r + 1.0) - 1.0) * 0.5);
    while (mu * (mu + 1) / 2 > r) --mu;
    while ((mu + 1) * (mu + 2) / 2 <= r) ++mu;
    const long long nu = r - mu * (mu + 1) / 2;
    const double* a = full + (mu * n + nu) * (long long)w;
    const double* b = full + (nu * n + mu) * (long long)w;
    double* out = packed + r * (long long)w;
    for (int c = threadIdx.x; c < w; c += blockDim.x) out[c] = 0.5 * (a[c] + b[c]);
  }
}

// sym[p][q] = (m[p][q] + m[q][p]) / 2
__global__ void symmetrize_kernel(const double* __restrict__ m, int x, double* __restrict__ sym) {
  const long long total = (long long)x * x;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long p = e / x, q = e - p * x;
    sym[e] = 0.5 * (m[e] + m[q * x + p]);
  }
}

struct DeviceFree {
  void operator()(void* p) const {
    if (p) cudaFree(p);
  }
};
using DevPtr = std::unique_ptr<void, DeviceFree>;

struct StreamGuard {
  cudaStream_t s = nullptr;
  ~StreamGuard() {
    if (s) {
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
    }
  }
};

int dev_alloc(DevPtr& out, size_t bytes, uint64_t& total, const char* what) {
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, std::max<size_t>(bytes, 8));
  if (e != cudaSuccess) return cuda_status(e, what);
  out.reset(p);
  total += bytes;
  return VQC_STATUS_SUCCESS;
}

int nfunc_of(int l, bool sph) { return sph ? 2 * l + 1 : (l + 1) * (l + 2) / 2; }

int run_gradient(Plan& plan, const double* xyz, const double* bar_a, const double* bar_m,
                 size_t maximum_bytes, size_t maximum_tile_elements, std::vector<double>& result,
                 vqc_df_gradient_resources& rec) {
  const long long n = plan.nao[0], x = plan.naux[0];
  const long long natom = plan.natom;
  const long long pairs = n * (n + 1) / 2;
  StreamGuard sg;
  cudaError_t e = cudaStreamCreateWithFlags(&sg.s, cudaStreamNonBlocking);
  if (e != cudaSuccess) return cuda_status(e, "df_gradient stream");
  const cudaStream_t st = sg.s;

  // fixed buffers: coordinates, gradient accumulator, the tile's molecule
  // view and its work lists
  const size_t fixed = (size_t)(2 * natom * 3) * sizeof(double) + sizeof(DevMol) +
                       plan.cls3c.size() * sizeof(ClassMol);
  if (fixed >= maximum_bytes)
    return fail(VQC_STATUS_OUT_OF_MEMORY, "df_gradient: maximum_bytes below the fixed buffers");
  DevPtr d_xyz, d_grad, d_mol, d_cms;
  uint64_t fixed_bytes = 0;
  int s = dev_alloc(d_xyz, natom * 3 * sizeof(double), fixed_bytes, "df_gradient xyz");
  if (!s) s = dev_alloc(d_grad, natom * 3 * sizeof(double), fixed_bytes, "df_gradient grad");
  if (!s) s = dev_alloc(d_mol, sizeof(DevMol), fixed_bytes, "df_gradient molecule view");
  if (!s) s = dev_alloc(d_cms, plan.cls3c.size() * sizeof(ClassMol), fixed_bytes, "df_gradient work");
  if (s) return s;
  uint64_t peak = fixed_bytes;  // device bytes held at once (metric and tiles do not overlap)
  if ((e = cudaMemcpyAsync(d_xyz.get(), xyz, natom * 3 * sizeof(double), cudaMemcpyHostToDevice, st)) ||
      (e = cudaMemsetAsync(d_grad.get(), 0, natom * 3 * sizeof(double), st)))
    return cuda_status(e, "df_gradient upload");
  rec.host_to_device_bytes += natom * 3 * sizeof(double);
  rec.uploads += 1;
  KernelArgs k = plan.args;
  k.xyz = static_cast<const double*>(d_xyz.get());
  k.grad = static_cast<double*>(d_grad.get());

  // metric channel: symmetric part of bar_m through the grad2c kernels
  if (bar_m) {
    const size_t mbytes = (size_t)(x * x) * sizeof(double);
    if (fixed + 2 * mbytes > maximum_bytes)
      return fail(VQC_STATUS_OUT_OF_MEMORY, "df_gradient: maximum_bytes cannot hold the X*X metric weights");
    DevPtr d_m, d_ms;
    uint64_t metric_bytes = 0;
    if ((s = dev_alloc(d_m, mbytes, metric_bytes, "df_gradient metric weights")) ||
        (s = dev_alloc(d_ms, mbytes, metric_bytes, "df_gradient metric weights")))
      return s;
    peak = std::max<uint64_t>(peak, fixed_bytes + metric_bytes);
    if ((e = cudaMemcpyAsync(d_m.get(), bar_m, mbytes, cudaMemcpyHostToDevice, st)))
      return cuda_status(e, "df_gradient metric upload");
    rec.host_to_device_bytes += mbytes;
    rec.uploads += 1;
    symmetrize_kernel<<<592, 256, 0, st>>>(static_cast<const double*>(d_m.get()), (int)x,
                                           static_cast<double*>(d_ms.get()));
    count_launch();
    if ((e = cudaGetLastError())) return cuda_status(e, "df_gradient symmetrize");
    KernelArgs km = k;
    km.w1 = static_cast<const double*>(d_ms.get());
    for (const ClassLaunch& cl : plan.cls2c) {
      if (!dispatch_grad2c(cl, km, plan.sph, st))
        return fail(VQC_STATUS_INVALID_ARGUMENT, "df_gradient: unsupported 2-centre class");
      count_launch();
      if ((e = cudaGetLastError())) return cuda_status(e, "df_gradient grad2c");
    }
    if ((e = cudaStreamSynchronize(st))) return cuda_status(e, "df_gradient metric");
    rec.stream_synchronizations += 1;
  }

  // 3-centre channel in auxiliary-shell column tiles
  if (bar_a) {
    const size_t per_col = (size_t)(n * n + pairs) * sizeof(double);
    long long wmax = (long long)((maximum_bytes - fixed) / per_col);
    if (maximum_tile_elements) wmax = std::min<long long>(wmax, (long long)(maximum_tile_elements / (size_t)(n * n)));
    wmax = std::min<long long>(wmax, x);
    const HostShells& ah = plan.aux_h;
    const int nsh = (int)ah.l.size();
    int widest = 0;
    for (int sh = 0; sh < nsh; ++sh) widest = std::max(widest, nfunc_of(ah.l[sh], plan.sph));
    if (wmax < widest)
      return fail(VQC_STATUS_OUT_OF_MEMORY,
                  "df_gradient: maximum_bytes / maximum_tile_elements cannot hold one auxiliary shell of weights");
    DevPtr d_full, d_packed;
    uint64_t tile_bytes = 0;
    if ((s = dev_alloc(d_full, (size_t)(n * n * wmax) * sizeof(double), tile_bytes, "df_gradient tile")) ||
        (s = dev_alloc(d_packed, (size_t)(pairs * wmax) * sizeof(double), tile_bytes, "df_gradient tile")))
      return s;
    peak = std::max<uint64_t>(peak, fixed_bytes + tile_bytes);
    rec.weight_tile_elements = (uint64_t)(n * n * wmax);
    std::vector<ClassMol> tile_cms(plan.cls3c.size());
    for (int s0 = 0; s0 < nsh;) {
      int s1 = s0, width = 0;
      while (s1 < nsh && width + nfunc_of(ah.l[s1], plan.sph) <= wmax) width += nfunc_of(ah.l[s1++], plan.sph);
      const long long p0 = ah.func_off[s0];
      // N*N rows of the tile's columns, then its packed symmetric part
      if ((e = cudaMemcpy2DAsync(d_full.get(), (size_t)width * sizeof(double), bar_a + p0,
                                 (size_t)x * sizeof(double), (size_t)width * sizeof(double),
                                 (size_t)(n * n), cudaMemcpyHostToDevice, st)))
        return cuda_status(e, "df_gradient tile upload");
      rec.host_to_device_bytes += (uint64_t)(n * n * width) * sizeof(double);
      rec.uploads += 1;
      pack_symmetric_tile_kernel<<<(unsigned)std::min<long long>(pairs, 148 * 16), 128, 0, st>>>(
          static_cast<const double*>(d_full.get()), (int)n, width, static_cast<double*>(d_packed.get()));
      count_launch();
      if ((e = cudaGetLastError())) return cuda_status(e, "df_gradient pack");
      // the molecule seen through the tile: row stride = tile width, column
      // origin = the tile's first auxiliary function
      DevMol view = plan.mols_h[0];
      view.naux = width;
      view.a_off = -p0;
      // work entries restricted to the tile's auxiliary shells
      std::vector<ClassLaunch> launches;
      int used = 0;
      for (size_t i = 0; i < plan.cls3c.size(); ++i) {
        const ClassLaunch& cl = plan.cls3c[i];
        const ClassMol& cm = plan.cls3c_host[i][0];
        const int lo = std::max(cm.aux_begin, s0), hi = std::min(cm.aux_begin + cm.naux, s1);
        if (lo >= hi) continue;
        const long long npair = cm.ntriples / cm.naux;
        const long long tri = npair * (hi - lo);
        const int per = slots3c(cl.la, cl.lb, cl.lc, plan.sph);
        tile_cms[used] = ClassMol{0, cm.pair_begin, lo, hi - lo, (int)tri, 0};
        ClassLaunch tl = cl;
        tl.cms = static_cast<const ClassMol*>(d_cms.get()) + used;
        tl.ncm = 1;
        tl.nblocks = (int)((tri + per - 1) / per);
        launches.push_back(tl);
        ++used;
      }
      if ((e = cudaMemcpyAsync(d_mol.get(), &view, sizeof(DevMol), cudaMemcpyHostToDevice, st)) ||
          (e = cudaMemcpyAsync(d_cms.get(), tile_cms.data(), used * sizeof(ClassMol),
                               cudaMemcpyHostToDevice, st)))
        return cuda_status(e, "df_gradient work upload");
      KernelArgs kt = k;
      kt.mols = static_cast<const DevMol*>(d_mol.get());
      kt.w1 = static_cast<const double*>(d_packed.get());
      for (const ClassLaunch& cl : launches) {
        if (!dispatch_grad3c(cl, kt, plan.sph, st))
          return fail(VQC_STATUS_INVALID_ARGUMENT, "df_gradient: unsupported 3-centre class");
        count_launch();
        if ((e = cudaGetLastError())) return cuda_status(e, "df_gradient grad3c");
      }
      // the host view / work entries and the tile buffers are reused next tile
      if ((e = cudaStreamSynchronize(st))) return cuda_status(e, "df_gradient tile");
      rec.stream_synchronizations += 1;
      rec.tiles += 1;
      s0 = s1;
    }
  }
  result.assign(natom * 3, 0.0);
  if ((e = cudaMemcpyAsync(result.data(), d_grad.get(), natom * 3 * sizeof(double),
                           cudaMemcpyDeviceToHost, st)) ||
      (e = cudaStreamSynchronize(st)))
    return cuda_status(e, "df_gradient download");
  rec.device_to_host_bytes += natom * 3 * sizeof(double);
  rec.stream_synchronizations += 1;
  rec.device_bytes = peak;
  for (double v : result)
    if (!std::isfinite(v)) return fail(VQC_STATUS_NUMERICAL_FAILURE, "df_gradient: non-finite gradient");
  return VQC_STATUS_SUCCESS;
}

}  // namespace
}  // namespace vqc

using namespace vqc;

extern "C" int vqc_df_gradient(const vqc_batch_desc* system, const double* xyz, const double* bar_a,
                               size_t count_a, const double* bar_m, size_t count_m, uint32_t schedule,
                               size_t maximum_bytes, size_t maximum_tile_elements, double* gradient,
                               size_t gradient_count, vqc_df_gradient_resources* resources) {
  try {
    if (!system || !xyz || !gradient || schedule > 1 || maximum_bytes == 0)
      return fail(VQC_STATUS_INVALID_ARGUMENT, "df_gradient: null argument, schedule > 1 or zero maximum_bytes");
    if (system->struct_size < sizeof(vqc_batch_desc) || system->abi_version != VQC_ABI_VERSION)
      return fail(VQC_STATUS_ABI_MISMATCH, "df_gradient: system descriptor struct_size/abi_version mismatch");
    if (resources && (resources->struct_size < sizeof(vqc_df_gradient_resources) ||
                      resources->abi_version != VQC_ABI_VERSION))
      return fail(VQC_STATUS_ABI_MISMATCH, "df_gradient: resources struct_size/abi_version mismatch");
    if (system->nmol != 1 || !system->mol_atom_offset || !system->mol_shell_offset || !system->mol_aux_offset)
      return fail(VQC_STATUS_INVALID_ARGUMENT, "df_gradient: the system descriptor must hold exactly one molecule");
    Plan plan;
    int st = plan.build(*system);
    if (st) return st;
    const size_t n = (size_t)plan.nao[0], x = (size_t)plan.naux[0];
    const size_t limit = ((size_t)-1) / sizeof(double);
    if (n > limit / n || n * n > limit / x || x > limit / x)
      return fail(VQC_STATUS_INVALID_ARGUMENT, "df_gradient: sizes overflow");
    if (count_a != n * n * x || count_m != x * x || gradient_count != 3 * (size_t)plan.natom)
      return fail(VQC_STATUS_INVALID_ARGUMENT,
                  "df_gradient: count_a must be N*N*X, count_m X*X and gradient_count 3*natom");
    vqc_df_gradient_resources rec{};
    rec.struct_size = sizeof(rec);
    rec.abi_version = VQC_ABI_VERSION;
    if (resources) *resources = rec;
    std::vector<double> result;
    st = run_gradient(plan, xyz, bar_a, bar_m, maximum_bytes, maximum_tile_elements, result, rec);
    if (st) return st;
    std::copy(result.begin(), result.end(), gradient);
    if (resources) *resources = rec;
    return VQC_STATUS_SUCCESS;
  } catch (const std::bad_alloc&) {
    return fail(VQC_STATUS_OUT_OF_MEMORY, "df_gradient: host allocation failed");
  } catch (...) {
    return fail(VQC_STATUS_NUMERICAL_FAILURE, "df_gradient: unexpected C++ exception");
  }
}
