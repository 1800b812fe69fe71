// Fused H.psi pass: star stencil + local potential + KB ket + Taylor/Horner
// epilogue + FP64 observables, over a packed (state-fastest) batch in the
// host's mesh point order.
#pragma once

#include "common.cuh"

namespace hpsi {

enum PassMode : int {
  PASS_APPLY = 0,   // out = H in
  PASS_HORNER = 1,  // out = psi0 + a * (H in)
};

struct PassArgs {
  CellBox box;
  const int *cell_src;    // per cell: source row to load, -1 zero, <= -2 periodic+phase
  const int *cell_row;    // per cell: own row (inner < np, boundary >= np) or -1
  const int *per_inner;   // boundary b -> inner image row (for encoded cells)
  const void *phase_corr; // complex (np_part - np), storage type of the batch
  int np;

  const void *in;         // stencil input batch
  long long in_ld;        // complex numbers per row
  long long in_rows;      // rows the input holds (the TMA fill's tensor extent)
  void *out;
  long long out_ld;
  const void *psi0;       // Horner: the untouched psi (pointwise term)
  long long psi0_ld;
  int mode;
  double a_re, a_im;      // Horner coefficient

  // per-axis weights, index d+4 for offset d; wx[4] holds the whole centre
  // weight, wy[4] = wz[4] = 0
  double wx[9], wy[9], wz[9];
  float wxf[9], wyf[9], wzf[9];  // the same weights rounded to FP32
  const double *v_cell;   // local potential in cell layout, or null
  double fld[3];          // laser: v += (fld . r), r = (cell + lo) * h
  const double *fld_scale_dev;  // optional device scalar multiplying fld

  // per-state observables of `in`: energy, norm, dipole partials
  double *obs;            // [ncta_xyz][obs_ld][3][2] (Kahan sum, compensation)
  int obs_ld;
  double obs_pol[3];      // dipole direction

  // density of the pass output (last Horner pass of a Taylor step):
  // rho_part[chunk][row] = sum over the chunk's states of w_i |out_i(row)|^2
  double *rho_part;       // [chunks][np], or null
  const double *rho_w;    // per state weight (ld entries)

  // TMA fill of the blocked pass: per (16 x 8 tile, cell plane) a mask whose
  // bit s marks star segment s (eight consecutive halo cells of one row) as
  // eight consecutive rows of the input; [tiles_y][seg_tiles_x][NZ]
  const unsigned long long *seg_mask;
  int seg_tiles_x;
  int *err;               // device status word of bounded waits (HPSI_ERR_TIMEOUT), or null

  const int2 *col_z;      // per (y, x) cell column: {first, last} z of its inner points
  const int4 *items;      // work items {tile x, tile y, first plane, end plane}
  int nitems;
  int chunks;             // state chunks per item (ld / SC)
  int zb;                 // output planes per item (at most)
};

// Kernel variant chosen for a pass.
struct PassShape {
  int sc;   // complex states per CTA
  int tx, ty, ry;
  int zb = 0;  // output planes per work item (0: chosen from the wave count)
  int unroll = 0;  // blocked pass: planes per unrolled group of the z march (1, 3 or 9)
  int blk = 0;     // 1: register-blocked real-lane pass (sc = its chunk, tiles 16 x 8)
  int rx = 0;      // blocked pass: cells per thread along x (ry along y)
  int cplx = 0;    // blocked pass: 1 = a thread owns a complex state, 0 = one real lane
  int tma = 0;     // blocked pass: contiguous halo runs filled by TMA box copies
  int mb = 0;      // blocked pass: stages handed over by mbarriers (split arrive / wait)
  int mma = 0;     // FP64 blocked pass with the x and y arms on the FP64 tensor cores (DMMA)
};

// Launch the fused pass for a storage type (double -> FP64, float -> FP32).
template <typename T>
hpsi_status launch_pass(PassArgs a, const PassShape &shape, cudaStream_t st);

// Tile edge (cells) of every pass kernel variant.
constexpr int PASS_TILE = 16;

// Systems of one grouped launch (their arguments travel as kernel parameters).
constexpr int GROUP_MAX = 48;
struct GroupArgs {
  PassArgs sys[GROUP_MAX];
  const int4 *units;   // {system, item, chunk, -}, most expensive first
  int nunits;
  int *counter;        // zeroed before every launch
};

// One persistent launch of the fused pass over several systems (no
// observables); sc must be a valid chunk for every system.
template <typename T>
hpsi_status launch_pass_group(const GroupArgs &g, int sc, int num_sms, cudaStream_t st);

}  // namespace hpsi
