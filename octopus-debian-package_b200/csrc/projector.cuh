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
  const double *pt64;    // the projector values in FP64 (tensor-core path)
  const double *scal64;  // the scales in FP64
  const void *psi;       // batch
  long long psi_ld;
  void *proj;            // projections [nprojections][proj_ld] complex
  long long proj_ld;
  int nprojections;
  int min_npoints;       // smallest sphere (bounds the K split)
  double *partial;       // split-K partials [ksplit][nprojections][proj_ld] complex, FP64
  const void *phase = nullptr;  // per sphere point complex phase (storage type), or null
};

struct KetArgs {
  int nk;                // covered rows
  const int *krows;      // covered row -> mesh row
  const int *kptr;       // nk + 1 offsets into ent
  const int4 *ent;       // {projector value offset, projection row, nproj, 0}
  const void *pt;        // projector values
  const void *proj;      // projections [nprojections][proj_ld] complex
  long long proj_ld;
  void *out;             // batch receiving the ket
  long long out_ld;
  int nst;
  int mode;              // 0: out += h; 1: out += a * h
  double a_re, a_im;
  const void *psi0;      // energy partials: Re(conj(psi0) h)
  long long psi0_ld;
  double *obs;           // [ket_row_blocks][obs_ld][2] or null
  int obs_ld;
  const void *phase = nullptr;  // per sphere point complex phase (storage type), or null
  // density of the final rows: rho_ket[blockIdx.x][covered row] = sum over the
  // CTA's states of w_i |out_i(row)|^2, or null
  double *rho_ket = nullptr;
  const double *rho_w = nullptr;
  // CTA rows of the launch, 0: ket_row_blocks(nk) (a launch that has the GPU
  // to itself); a grouped step gives each of its concurrent kets fewer
  int row_blocks = 0;
};

int bra_ksplit(const ProjArgs &p, int num_sms);
int ket_row_blocks(int nk);

template <typename T>
hpsi_status launch_bra(const ProjArgs &p, bool use_tensor, int ksplit, cudaStream_t st);
template <typename T>
hpsi_status launch_ket(const KetArgs &k, cudaStream_t st);

}  // namespace hpsi
