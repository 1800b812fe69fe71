// Handle layouts behind the opaque C types of hpsi.h.
#pragma once

#include <map>
#include <vector>

#include "common.cuh"
#include "stencil.cuh"

namespace hpsi {

hpsi_status dev_alloc(void **p, size_t bytes);
struct PassArgs;
struct PassShape;
// TMA fill of a blocked pass: segment masks, status word and input extent in
// `a`; clears shape.tma where the load map has no table (periodic images)
hpsi_status prepare_tma(hpsi_hamiltonian *h, const int *src_map, long long in_rows, PassShape &shape, PassArgs &a);
void dev_free(void *p);
bool is_device_ptr(const void *p);

// Times the kernels launched in its scope on `st` when profiling is enabled.
class ProfScope {
 public:
  ProfScope(const char *label, cudaStream_t st);
  ~ProfScope();

 private:
  cudaStream_t st_;
  long idx_ = -1;
};

// Grow-only device buffer owned by a handle.
struct Workspace {
  void *ptr = nullptr;
  size_t size = 0;
  hpsi_status ensure(size_t bytes);
  void release();
};

}  // namespace hpsi

struct hpsi_mesh {
  int np = 0, np_part = 0, order = 4, periodic = 0;
  hpsi::CellBox box{};
  std::vector<int> per_inner_h;
  std::vector<int> cell_of_row_h;
  int *d_cell_row = nullptr;   // own row of each cell, -1 outside the mesh
  int *d_src_raw = nullptr;    // load map: every mesh point as stored
  int *d_src_zero = nullptr;   // load map: zero boundary condition
  int *d_src_per = nullptr;    // load map: periodic images
  int *d_per_inner = nullptr;
  int *d_cell_of_row = nullptr;
  int device = 0, num_sms = 148;
  hpsi::Workspace scratch, scratch2, stage_in, stage_out;
  // z range {first, last} (cells) of the inner points of each 16x16 tile
  // column, and of each 16x8 tile column (the blocked pass)
  int tiles_x = 0, tiles_y = 0, tiles_y8 = 0;
  std::vector<int2> tile_z, tile_z8;
  long long column_planes = 0;          // sum of the tile z extents
  // work list per (z block depth, tile height): key 2 * zb + (height == 8)
  std::map<int, std::pair<int4 *, int>> items;
  // z block depth of a single-system blocked pass, per state chunk count
  mutable std::map<int, int> zb_single;
  // domain-parallel meshes: rows [ghost_first, ghost_first + ghost_count) hold
  // other partitions' points; work lists split into the tiles/planes whose
  // stencil reads no ghost row (part 1) and the rest (part 2), per (zb, ty)
  int ghost_first = 0, ghost_count = 0;
  std::map<int, std::pair<int4 *, int>> items_part;
  // TMA fill: own row of every cell (host), and per load map the device table
  // of contiguous star segments (PassArgs::seg_mask)
  std::vector<int> cell_row_h;
  std::map<const int *, unsigned long long *> seg_masks;
  int2 *d_col_z = nullptr;  // per (y, x) cell column: z range of its inner points
};

struct hpsi_hamiltonian {
  hpsi_mesh *mesh = nullptr;
  bool have_kinetic = false;
  double wx[9] = {0}, wy[9] = {0}, wz[9] = {0};
  double *d_vcell = nullptr;
  double fld[3] = {0, 0, 0};
  double pol[3] = {0, 0, 1};
  bool have_pol = false;
  double *d_phase = nullptr;
  float *d_phase_f = nullptr;
  int *d_src_phase = nullptr;
  // KB projectors
  int nmat = 0, nprojections = 0, max_nproj = 0;
  int4 *d_mat = nullptr;
  int *d_proj_row = nullptr, *d_map = nullptr;
  double *d_pt = nullptr, *d_scal = nullptr;
  float *d_pt_f = nullptr, *d_scal_f = nullptr;
  // rows covered by at least one sphere: krows[nk], entries kptr[nk+1] -> kb_ent
  int nk = 0, min_npoints = 0;
  int *d_krows = nullptr, *d_kptr = nullptr;
  int *d_kidx = nullptr;  // per inner row: its index among the covered rows, or -1
  int4 *d_kb_ent = nullptr;
  // projector phases (k != 0): one complex number per sphere point, or null
  long long kb_npts = 0;
  std::vector<int> kb_npoints_h;  // sphere points of each matrix
  double *d_kb_phase = nullptr;
  float *d_kb_phase_f = nullptr;
  bool use_tensor_bra = true;
  // autotuned pass shape per storage type (valid for batches of width ld)
  struct Tuned {
    long long ld = -1;
    hpsi::PassShape shape{};
    double ms = 0.0;
  } tuned[2];
  const double *fld_scale_dev = nullptr;  // set while a TD run replays steps
  // side stream of the KB bra (forked from the caller's stream, joined before the ket)
  bool overlap_bra = true;
  bool fuse_density = false;  // hpsi_taylor_step_density: density in the last pass (slower, kept for measurement)
  cudaStream_t bra_stream = nullptr;
  cudaEvent_t bra_fork = nullptr, bra_join = nullptr;
  // the pass of an H psi with a side-stream bra runs on a high-priority stream
  // of its own, so that pending pass CTAs take freed SMs before bra CTAs
  bool prio_pass = true;
  cudaStream_t pass_stream = nullptr;
  cudaEvent_t pass_join = nullptr;
  hpsi_status ensure_bra_stream();
  cudaStream_t capture_stream = nullptr;  // graph capture / replay stream of TD runs
  cudaEvent_t capture_event = nullptr;
  // host-batch pipeline: copy-in and copy-out streams, per-buffer events
  // {copied in, computed, copied out} x 2 buffers, and the slab buffers
  cudaStream_t xfer_in = nullptr, xfer_out = nullptr;
  cudaEvent_t xev[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  hpsi::Workspace slab_in, slab_out;
  // workspaces
  hpsi::Workspace u[2], projbuf, bra_partial, obsbuf, ketobs, small, tdbuf, adjbuf;
  hpsi::Workspace lzbuf, lzsmall;
  hpsi::Workspace vstage;  // host potential staged for hpsi_hamiltonian_update_vloc
  hpsi::Workspace adjstep, vjpbuf;  // per-step adjoint scratch, field VJP partials
  hpsi::Workspace rhobuf;  // fused density: weights, pass and ket partials
  int *d_err = nullptr;     // status word of the passes' bounded waits  // Lanczos: Krylov vectors, reductions and coefficients
  void proj_free();
};
