// C ABI and the batch plan: validates the ragged batch, lays out per-molecule
// offsets, builds the angular-momentum class work lists and uploads them once.
//
// Reference counterparts: generativeqc_batch_prepare (src/api/c_api_batch.cpp:25)
// builds a FleetPlan that buckets systems (src/scf/fleet.cpp:27-35,131); here
// every molecule of the batch shares one plan and one launch per class.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "vqc_df.h"
#include "vqc_kernels.cuh"
#include "vqc_plan.hpp"

namespace vqc {

thread_local std::string g_last_error;
std::atomic<unsigned long long> g_launches{0};

// tuning knobs: process-wide, read at launch time; values are checked against
// each knob's range when set
static std::atomic<int> g_tune[VQC_TUNE_COUNT] = {0, 2};
static const int kTuneMin[VQC_TUNE_COUNT] = {0, 1};
static const int kTuneMax[VQC_TUNE_COUNT] = {0, 64};

int tune_value(int knob) {
  return (knob > 0 && knob < VQC_TUNE_COUNT) ? g_tune[knob].load(std::memory_order_relaxed) : 0;
}

int fail(int status, const std::string& msg) {
  g_last_error = msg;
  return status;
}

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

int cuda_status(cudaError_t e, const char* where) {
  if (e == cudaSuccess) return VQC_STATUS_SUCCESS;
  return fail(e == cudaErrorMemoryAllocation ? VQC_STATUS_OUT_OF_MEMORY : VQC_STATUS_CUDA_ERROR,
              std::string(where) + ": " + cudaGetErrorString(e));
}

static int nfunc(int l, bool sph) { return sph ? 2 * l + 1 : (l + 1) * (l + 2) / 2; }

template <typename T>
static int upload(DeviceBuffers& owned, const std::vector<T>& h, T** d) {
  *d = nullptr;
  if (h.empty()) return VQC_STATUS_SUCCESS;
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, h.size() * sizeof(T));
  if (e != cudaSuccess) return cuda_status(e, "plan upload");
  owned.push_back(p);
  e = cudaMemcpy(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_status(e, "plan upload");
  *d = static_cast<T*>(p);
  return VQC_STATUS_SUCCESS;
}

Plan::~Plan() {
  for (void* p : owned) cudaFree(p);
}

static int build_shells(const int32_t* l, const int32_t* atom, const int32_t* nprim,
                        const int32_t* poff, int32_t nprim_total, const int32_t* mol_off,
                        const int32_t* mol_atom_off, int nmol, bool sph, HostShells& hs,
                        std::vector<int>& nfunc_mol, const char* what) {
  int nshell = mol_off[nmol];
  hs.l.assign(l, l + nshell);
  hs.atom.assign(atom, atom + nshell);
  hs.nprim.assign(nprim, nprim + nshell);
  hs.prim_off.assign(poff, poff + nshell);
  hs.func_off.resize(nshell);
  nfunc_mol.assign(nmol, 0);
  for (int m = 0; m < nmol; ++m) {
    if (mol_off[m + 1] < mol_off[m]) return fail(VQC_STATUS_INVALID_ARGUMENT, std::string(what) + ": shell offsets decrease");
    int f = 0;
    for (int s = mol_off[m]; s < mol_off[m + 1]; ++s) {
      if (l[s] < 0 || l[s] > kMaxKernelL)
        return fail(VQC_STATUS_INVALID_ARGUMENT, std::string(what) + ": angular momentum outside 0..3");
      if (nprim[s] <= 0 || poff[s] < 0 || poff[s] + nprim[s] > nprim_total)
        return fail(VQC_STATUS_INVALID_ARGUMENT, std::string(what) + ": primitive range");
      if (atom[s] < mol_atom_off[m] || atom[s] >= mol_atom_off[m + 1])
        return fail(VQC_STATUS_INVALID_ARGUMENT, std::string(what) + ": shell atom outside its molecule");
      hs.func_off[s] = f;
      f += nfunc(l[s], sph);
    }
    nfunc_mol[m] = f;
  }
  return VQC_STATUS_SUCCESS;
}

int Plan::build(const vqc_batch_desc& d) {
  nmol = d.nmol;
  sph = d.spherical != 0;
  mol_shell_off.assign(d.mol_shell_offset, d.mol_shell_offset + d.nmol + 1);
  natom = d.mol_atom_offset[nmol];
  int st = build_shells(d.shell_l, d.shell_atom, d.shell_nprim, d.shell_prim_off, d.nprim,
                        d.mol_shell_offset, d.mol_atom_offset, nmol, sph, orb_h, nao, "orbital");
  if (st) return st;
  st = build_shells(d.aux_l, d.aux_atom, d.aux_nprim, d.aux_prim_off, d.naux_prim,
                    d.mol_aux_offset, d.mol_atom_offset, nmol, sph, aux_h, naux, "auxiliary");
  if (st) return st;
  for (int m = 0; m < nmol; ++m)
    for (int s = d.mol_aux_offset[m] + 1; s < d.mol_aux_offset[m + 1]; ++s)
      if (d.aux_l[s] < d.aux_l[s - 1])
        return fail(VQC_STATUS_INVALID_ARGUMENT, "auxiliary shells must be sorted by l per molecule");
  // molecule table
  mols_h.resize(nmol);
  long long mo = 0, me = 0, ao = 0;
  for (int m = 0; m < nmol; ++m) {
    DevMol& dm = mols_h[m];
    dm.nao = nao[m];
    dm.naux = naux[m];
    dm.atom_off = d.mol_atom_offset[m];
    dm.natom = d.mol_atom_offset[m + 1] - d.mol_atom_offset[m];
    if (dm.natom <= 0 || dm.nao <= 0 || dm.naux <= 0)
      return fail(VQC_STATUS_INVALID_ARGUMENT, "molecule without atoms or functions");
    dm.mat_off = mo;
    dm.met_off = me;
    dm.a_off = ao;
    mo += (long long)dm.nao * dm.nao;
    me += (long long)dm.naux * dm.naux;
    ao += (long long)dm.nao * (dm.nao + 1) / 2 * dm.naux;
  }
  mat_total = mo;
  met_total = me;
  a_total = ao;

  // pair lists per (la >= lb) class, shared by 1e and 3c; 2c pairs of aux shells
  std::vector<std::vector<int2>> pl(16), pl2(16);
  std::vector<std::vector<int>> pbeg(16, std::vector<int>(nmol)), pcnt(16, std::vector<int>(nmol));
  std::vector<std::vector<int>> qbeg(16, std::vector<int>(nmol)), qcnt(16, std::vector<int>(nmol));
  for (int m = 0; m < nmol; ++m) {
    for (int c = 0; c < 16; ++c) {
      pbeg[c][m] = (int)pl[c].size();
      qbeg[c][m] = (int)pl2[c].size();
    }
    for (int a = d.mol_shell_offset[m]; a < d.mol_shell_offset[m + 1]; ++a)
      for (int b = d.mol_shell_offset[m]; b <= a; ++b) {
        int la = d.shell_l[a], lb = d.shell_l[b];
        int2 pr = la >= lb ? make_int2(a, b) : make_int2(b, a);
        pl[std::max(la, lb) * 4 + std::min(la, lb)].push_back(pr);
      }
    for (int a = d.mol_aux_offset[m]; a < d.mol_aux_offset[m + 1]; ++a)
      for (int b = d.mol_aux_offset[m]; b <= a; ++b) {
        int la = d.aux_l[a], lb = d.aux_l[b];
        int2 pr = la >= lb ? make_int2(a, b) : make_int2(b, a);
        pl2[std::max(la, lb) * 4 + std::min(la, lb)].push_back(pr);
      }
    for (int c = 0; c < 16; ++c) {
      pcnt[c][m] = (int)pl[c].size() - pbeg[c][m];
      qcnt[c][m] = (int)pl2[c].size() - qbeg[c][m];
    }
  }
  // aux ranges per l per molecule
  std::vector<std::vector<int>> abeg(4, std::vector<int>(nmol, 0)), acnt(4, std::vector<int>(nmol, 0));
  for (int m = 0; m < nmol; ++m)
    for (int s = d.mol_aux_offset[m + 1] - 1; s >= d.mol_aux_offset[m]; --s) {
      abeg[d.aux_l[s]][m] = s;
      acnt[d.aux_l[s]][m]++;
    }

  st = upload(owned, orb_h.l, &dorb_l);
  if (!st) st = upload(owned, orb_h.atom, &dorb_atom);
  if (!st) st = upload(owned, orb_h.nprim, &dorb_nprim);
  if (!st) st = upload(owned, orb_h.prim_off, &dorb_poff);
  if (!st) st = upload(owned, orb_h.func_off, &dorb_foff);
  if (!st) st = upload(owned, std::vector<double>(d.prim_exp, d.prim_exp + d.nprim), &dorb_exp);
  if (!st) st = upload(owned, std::vector<double>(d.prim_coef, d.prim_coef + d.nprim), &dorb_coef);
  if (!st) st = upload(owned, aux_h.l, &daux_l);
  if (!st) st = upload(owned, aux_h.atom, &daux_atom);
  if (!st) st = upload(owned, aux_h.nprim, &daux_nprim);
  if (!st) st = upload(owned, aux_h.prim_off, &daux_poff);
  if (!st) st = upload(owned, aux_h.func_off, &daux_foff);
  if (!st) st = upload(owned, std::vector<double>(d.aux_exp, d.aux_exp + d.naux_prim), &daux_exp);
  if (!st) st = upload(owned, std::vector<double>(d.aux_coef, d.aux_coef + d.naux_prim), &daux_coef);
  if (!st) st = upload(owned, std::vector<double>(d.atom_charge, d.atom_charge + natom), &dcharge);
  if (!st) st = upload(owned, mols_h, &dmols);
  if (st) return st;
  args.orb = DevBasis{dorb_l, dorb_atom, dorb_nprim, dorb_poff, dorb_foff, dorb_exp, dorb_coef};
  args.aux = DevBasis{daux_l, daux_atom, daux_nprim, daux_poff, daux_foff, daux_exp, daux_coef};
  args.charge = dcharge;
  args.mols = dmols;

  int2* dpairs[16] = {nullptr};
  int2* dpairs2[16] = {nullptr};
  for (int c = 0; c < 16; ++c) {
    if ((st = upload(owned, pl[c], &dpairs[c]))) return st;
    if ((st = upload(owned, pl2[c], &dpairs2[c]))) return st;
  }
  auto add_class = [&](std::vector<ClassLaunch>& list, int la, int lb, int lc, const int2* pairs,
                       std::vector<ClassMol>& cms, int per_block) -> int {
    if (cms.empty()) return VQC_STATUS_SUCCESS;
    int nb = 0;
    for (auto& c : cms) {
      c.chunk_begin = nb;
      long long blocks = (c.ntriples + per_block - 1) / per_block;
      if (nb + blocks > 0x7fffffffLL) return fail(VQC_STATUS_INVALID_ARGUMENT, "batch too large for one launch");
      nb += (int)blocks;
    }
    ClassMol* dcm = nullptr;
    int s2 = upload(owned, cms, &dcm);
    if (s2) return s2;
    list.push_back(ClassLaunch{la, lb, lc, pairs, dcm, (int)cms.size(), nb});
    return VQC_STATUS_SUCCESS;
  };
  for (int la = 0; la <= kMaxKernelL; ++la)
    for (int lb = 0; lb <= la; ++lb) {
      int c = la * 4 + lb;
      std::vector<ClassMol> one;
      for (int m = 0; m < nmol; ++m)
        if (pcnt[c][m]) one.push_back(ClassMol{m, pbeg[c][m], 0, 0, pcnt[c][m], 0});
      if ((st = add_class(cls1e, la, lb, 0, dpairs[c], one, 128))) return st;
      for (int lc = 0; lc <= kMaxKernelL; ++lc) {
        std::vector<ClassMol> cm3;
        for (int m = 0; m < nmol; ++m) {
          long long tri = (long long)pcnt[c][m] * acnt[lc][m];
          if (!tri) continue;
          if (tri > 0x7fffffffLL) return fail(VQC_STATUS_INVALID_ARGUMENT, "molecule too large for the 3-centre work list");
          cm3.push_back(ClassMol{m, pbeg[c][m], abeg[lc][m], acnt[lc][m], (int)tri, 0});
        }
        if ((st = add_class(cls3c, la, lb, lc, dpairs[c], cm3, slots3c(la, lb, lc, sph)))) return st;
        if (!cm3.empty()) cls3c_host.push_back(cm3);
      }
      std::vector<ClassMol> cm2;
      for (int m = 0; m < nmol; ++m)
        if (qcnt[c][m]) cm2.push_back(ClassMol{m, qbeg[c][m], 0, 0, qcnt[c][m], 0});
      if ((st = add_class(cls2c, la, 0, lb, dpairs2[c], cm2, slots2c(lb)))) return st;
    }
  // scratch of the bounded row tiles: one molecule view, one entry per class
  std::vector<DevMol> view(1);
  if ((st = upload(owned, view, &dtile_mol))) return st;
  std::vector<ClassMol> tcms(std::max<size_t>(1, cls3c.size()));
  if ((st = upload(owned, tcms, &dtile_cms))) return st;
  return VQC_STATUS_SUCCESS;
}

}  // namespace vqc

using namespace vqc;

#define VQC_GUARD_BEGIN try {
#define VQC_GUARD_END                                                   \
  }                                                                     \
  catch (const std::bad_alloc&) {                                       \
    return fail(VQC_STATUS_OUT_OF_MEMORY, "host allocation failed");    \
  }                                                                     \
  catch (...) {                                                         \
    return fail(VQC_STATUS_NUMERICAL_FAILURE, "unexpected C++ exception"); \
  }

extern "C" {

const char* vqc_last_error(void) { return g_last_error.c_str(); }
uint32_t vqc_abi_version(void) { return VQC_ABI_VERSION; }
uint64_t vqc_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

int vqc_tune_set(int32_t knob, int32_t value) {
  if (knob <= 0 || knob >= VQC_TUNE_COUNT || value < kTuneMin[knob] || value > kTuneMax[knob])
    return fail(VQC_STATUS_INVALID_ARGUMENT, "tune_set: unknown knob or value out of range");
  g_tune[knob].store(value, std::memory_order_relaxed);
  return VQC_STATUS_SUCCESS;
}

int vqc_tune_get(int32_t knob, int32_t* value) {
  if (knob <= 0 || knob >= VQC_TUNE_COUNT || !value)
    return fail(VQC_STATUS_INVALID_ARGUMENT, "tune_get: unknown knob");
  *value = g_tune[knob].load(std::memory_order_relaxed);
  return VQC_STATUS_SUCCESS;
}

int vqc_plan_create(const vqc_batch_desc* desc, vqc_plan** out) {
  VQC_GUARD_BEGIN
  if (!desc || !out) return fail(VQC_STATUS_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  if (desc->struct_size < sizeof(vqc_batch_desc) || desc->abi_version != VQC_ABI_VERSION)
    return fail(VQC_STATUS_ABI_MISMATCH, "descriptor struct_size/abi_version mismatch");
  if (desc->nmol <= 0 || !desc->mol_atom_offset || !desc->mol_shell_offset || !desc->mol_aux_offset)
    return fail(VQC_STATUS_INVALID_ARGUMENT, "empty batch");
  Plan* p = new Plan();
  int st = p->build(*desc);
  if (st) {
    delete p;
    return st;
  }
  *out = reinterpret_cast<vqc_plan*>(p);
  return VQC_STATUS_SUCCESS;
  VQC_GUARD_END
}

int vqc_plan_destroy(vqc_plan* plan) {
  delete reinterpret_cast<Plan*>(plan);
  return VQC_STATUS_SUCCESS;
}

int vqc_plan_totals(const vqc_plan* plan, int64_t* mat_total, int64_t* met_total, int64_t* a_total,
                    int32_t* natom_total) {
  if (!plan) return fail(VQC_STATUS_INVALID_ARGUMENT, "null plan");
  const Plan* p = reinterpret_cast<const Plan*>(plan);
  if (mat_total) *mat_total = p->mat_total;
  if (met_total) *met_total = p->met_total;
  if (a_total) *a_total = p->a_total;
  if (natom_total) *natom_total = p->natom;
  return VQC_STATUS_SUCCESS;
}

int vqc_plan_molecule(const vqc_plan* plan, int32_t index, vqc_molecule_info* info) {
  if (!plan || !info) return fail(VQC_STATUS_INVALID_ARGUMENT, "null argument");
  const Plan* p = reinterpret_cast<const Plan*>(plan);
  if (index < 0 || index >= p->nmol) return fail(VQC_STATUS_INVALID_ARGUMENT, "molecule index");
  const DevMol& m = p->mols_h[index];
  info->nao = m.nao;
  info->naux = m.naux;
  info->natom = m.natom;
  info->atom_offset = m.atom_off;
  info->mat_offset = m.mat_off;
  info->met_offset = m.met_off;
  info->a_offset = m.a_off;
  return VQC_STATUS_SUCCESS;
}

static int run_classes(Plan* p, const std::vector<ClassLaunch>& list,
                       bool (*dispatch)(const ClassLaunch&, const KernelArgs&, bool, cudaStream_t),
                       const KernelArgs& k, cudaStream_t st, const char* what) {
  for (const ClassLaunch& cl : list) {
    if (!dispatch(cl, k, p->sph, st))
      return fail(VQC_STATUS_INVALID_ARGUMENT, std::string(what) + ": unsupported class");
    g_launches.fetch_add(1, std::memory_order_relaxed);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_status(e, what);
  }
  return VQC_STATUS_SUCCESS;
}

int vqc_int1e(vqc_plan* plan, const double* xyz, double* s, double* t, double* v, void* stream) {
  VQC_GUARD_BEGIN
  if (!plan || !xyz || !s || !t || !v) return fail(VQC_STATUS_INVALID_ARGUMENT, "null argument");
  Plan* p = reinterpret_cast<Plan*>(plan);
  KernelArgs k = p->args;
  k.xyz = xyz;
  k.out = s;
  k.out2 = t;
  k.out3 = v;
  return run_classes(p, p->cls1e, dispatch_int1e, k, (cudaStream_t)stream, "int1e");
  VQC_GUARD_END
}

int vqc_int2c(vqc_plan* plan, const double* xyz, double* metric, void* stream) {
  VQC_GUARD_BEGIN
  if (!plan || !xyz || !metric) return fail(VQC_STATUS_INVALID_ARGUMENT, "null argument");
  Plan* p = reinterpret_cast<Plan*>(plan);
  KernelArgs k = p->args;
  k.xyz = xyz;
  k.out = metric;
  return run_classes(p, p->cls2c, dispatch_int2c, k, (cudaStream_t)stream, "int2c");
  VQC_GUARD_END
}

int vqc_int3c(vqc_plan* plan, const double* xyz, double* a_packed, void* stream) {
  VQC_GUARD_BEGIN
  if (!plan || !xyz || !a_packed) return fail(VQC_STATUS_INVALID_ARGUMENT, "null argument");
  Plan* p = reinterpret_cast<Plan*>(plan);
  KernelArgs k = p->args;
  k.xyz = xyz;
  k.out = a_packed;
  return run_classes(p, p->cls3c, dispatch_int3c, k, (cudaStream_t)stream, "int3c");
  VQC_GUARD_END
}

int vqc_int3c_rows(vqc_plan* plan, const double* xyz, int32_t mol, int32_t shell_begin,
                   int32_t shell_end, double* rows, void* stream) {
  VQC_GUARD_BEGIN
  if (!plan || !xyz || !rows) return fail(VQC_STATUS_INVALID_ARGUMENT, "null argument");
  Plan* p = reinterpret_cast<Plan*>(plan);
  if (mol < 0 || mol >= p->nmol) return fail(VQC_STATUS_INVALID_ARGUMENT, "int3c_rows: molecule index");
  const int s0 = p->mol_shell_off[mol], s1 = p->mol_shell_off[mol + 1];
  if (shell_begin < 0 || shell_end <= shell_begin || s0 + shell_end > s1)
    return fail(VQC_STATUS_INVALID_ARGUMENT, "int3c_rows: shell range outside the molecule");
  const int a0 = s0 + shell_begin, a1 = s0 + shell_end;
  const long long f0 = p->orb_h.func_off[a0];
  const long long naux = p->mols_h[mol].naux;
  // the molecule seen through the tile: packed rows counted from the tile's first row
  DevMol view = p->mols_h[mol];
  view.a_off = -(f0 * (f0 + 1) / 2) * naux;
  // pairs (a, b <= a) of a class are listed in order of a, so the tile's pairs
  // (a in [a0, a1)) are one contiguous run per class: count the pairs before it
  auto class_of = [&](int a, int b) {
    const int la = p->orb_h.l[a], lb = p->orb_h.l[b];
    return std::max(la, lb) * 4 + std::min(la, lb);
  };
  int before[16] = {0}, inside[16] = {0};
  for (int a = s0; a < a1; ++a)
    for (int b = s0; b <= a; ++b) (a < a0 ? before : inside)[class_of(a, b)]++;
  std::vector<ClassMol> cms;
  std::vector<ClassLaunch> launches;
  for (size_t i = 0; i < p->cls3c.size(); ++i) {
    const ClassLaunch& cl = p->cls3c[i];
    const int c = cl.la * 4 + cl.lb;
    if (!inside[c]) continue;
    const ClassMol* cm = nullptr;
    for (const ClassMol& e : p->cls3c_host[i])
      if (e.mol == mol) cm = &e;
    if (!cm) continue;  // no auxiliary shell of this class's l in the molecule
    const long long tri = (long long)inside[c] * cm->naux;
    const int per = slots3c(cl.la, cl.lb, cl.lc, p->sph);
    ClassLaunch tl = cl;
    tl.cms = p->dtile_cms + cms.size();
    tl.ncm = 1;
    tl.nblocks = (int)((tri + per - 1) / per);
    cms.push_back(ClassMol{0, cm->pair_begin + before[c], cm->aux_begin, cm->naux, (int)tri, 0});
    launches.push_back(tl);
  }
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e;
  if ((e = cudaMemcpyAsync(p->dtile_mol, &view, sizeof(DevMol), cudaMemcpyHostToDevice, st)))
    return cuda_status(e, "int3c_rows view upload");
  if (!cms.empty() &&
      (e = cudaMemcpyAsync(p->dtile_cms, cms.data(), cms.size() * sizeof(ClassMol),
                           cudaMemcpyHostToDevice, st)))
    return cuda_status(e, "int3c_rows work upload");
  KernelArgs k = p->args;
  k.xyz = xyz;
  k.out = rows;
  k.mols = p->dtile_mol;
  return run_classes(p, launches, dispatch_int3c, k, st, "int3c_rows");
  VQC_GUARD_END
}

int vqc_grad3c(vqc_plan* plan, const double* xyz, const double* abar_packed, double* grad,
               void* stream) {
  VQC_GUARD_BEGIN
  if (!plan || !xyz || !abar_packed || !grad) return fail(VQC_STATUS_INVALID_ARGUMENT, "null argument");
  Plan* p = reinterpret_cast<Plan*>(plan);
  KernelArgs k = p->args;
  k.xyz = xyz;
  k.w1 = abar_packed;
  k.grad = grad;
  return run_classes(p, p->cls3c, dispatch_grad3c, k, (cudaStream_t)stream, "grad3c");
  VQC_GUARD_END
}

int vqc_grad2c(vqc_plan* plan, const double* xyz, const double* mbar, double* grad, void* stream) {
  VQC_GUARD_BEGIN
  if (!plan || !xyz || !mbar || !grad) return fail(VQC_STATUS_INVALID_ARGUMENT, "null argument");
  Plan* p = reinterpret_cast<Plan*>(plan);
  KernelArgs k = p->args;
  k.xyz = xyz;
  k.w1 = mbar;
  k.grad = grad;
  return run_classes(p, p->cls2c, dispatch_grad2c, k, (cudaStream_t)stream, "grad2c");
  VQC_GUARD_END
}

int vqc_grad1e(vqc_plan* plan, const double* xyz, const double* dens, const double* wdens,
               double* grad, void* stream) {
  VQC_GUARD_BEGIN
  if (!plan || !xyz || !dens || !wdens || !grad) return fail(VQC_STATUS_INVALID_ARGUMENT, "null argument");
  Plan* p = reinterpret_cast<Plan*>(plan);
  KernelArgs k = p->args;
  k.xyz = xyz;
  k.w1 = dens;
  k.w2 = wdens;
  k.grad = grad;
  return run_classes(p, p->cls1e, dispatch_grad1e, k, (cudaStream_t)stream, "grad1e");
  VQC_GUARD_END
}

}  // extern "C"
