// KB projector bra kernels (see projector.cu).
#pragma once

#include "common.cuh"

namespace hpsi {

struct ProjArgs {
  int nmat;
  int max_nproj;
  const int4 *mat;       // per matrix: {npoints, nproj, map offset, projector value offset}
  const int *proj_row;   // per matrix: first projection row
  const int *map;        // sphere point -> mesh row
  const void *pt;        // projector values, projector index fastest per point
  const void *scal;      // per projector scale (storage type)
  const void *psi;       // batch
  long long psi_ld;
  void *proj;            // projections [nprojections][proj_ld] complex
  long long proj_ld;
};

template <typename T>
hpsi_status launch_bra(const ProjArgs &p, bool use_tensor, cudaStream_t st);

}  // namespace hpsi
