// Host-side plan object behind the opaque vqc_plan handle.
#pragma once

#include <string>
#include <vector>

#include "vqc_df.h"
#include "vqc_kernels.cuh"

namespace vqc {

constexpr int kMaxKernelL = 3;  // angular momentum the dispatch tables instantiate

using DeviceBuffers = std::vector<void*>;

struct HostShells {
  std::vector<int> l, atom, nprim, prim_off, func_off;
};

struct Plan {
  int nmol = 0;
  bool sph = true;
  int natom = 0;
  std::vector<int> nao, naux;
  std::vector<DevMol> mols_h;
  HostShells orb_h, aux_h;
  long long mat_total = 0, met_total = 0, a_total = 0;

  DeviceBuffers owned;
  int *dorb_l = nullptr, *dorb_atom = nullptr, *dorb_nprim = nullptr, *dorb_poff = nullptr,
      *dorb_foff = nullptr;
  double *dorb_exp = nullptr, *dorb_coef = nullptr;
  int *daux_l = nullptr, *daux_atom = nullptr, *daux_nprim = nullptr, *daux_poff = nullptr,
      *daux_foff = nullptr;
  double *daux_exp = nullptr, *daux_coef = nullptr;
  double* dcharge = nullptr;
  DevMol* dmols = nullptr;
  KernelArgs args{};

  std::vector<ClassLaunch> cls1e, cls2c, cls3c;
  // host copies of the per-molecule work entries of each cls3c launch (the
  // tiled gradient entry re-slices them by auxiliary shell range)
  std::vector<std::vector<ClassMol>> cls3c_host;
  // orbital shell range of every molecule (global shell indices), and a
  // device scratch (one molecule view + one work entry per 3-centre class)
  // for the bounded row tiles of vqc_int3c_rows
  std::vector<int> mol_shell_off;
  DevMol* dtile_mol = nullptr;
  ClassMol* dtile_cms = nullptr;

  int build(const vqc_batch_desc& d);
  ~Plan();
};

// current value of a tuning knob (vqc_tune_set; defaults in capi.cu)
int tune_value(int knob);

int fail(int status, const std::string& msg);
void count_launch();
int cuda_status(cudaError_t e, const char* where);

}  // namespace vqc
