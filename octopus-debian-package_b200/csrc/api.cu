// C ABI of the hpsi library: handles, validation, workspace and dispatch.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <queue>
#include <vector>

#include "api_internal.cuh"
#include "projector.cuh"
#include "reduce.cuh"
#include "stencil.cuh"
#include "stencil_blk.cuh"

namespace hpsi {

std::atomic<int64_t> g_launches{0};
static thread_local std::string t_last_error;
void set_error(const std::string &msg) { t_last_error = msg; }

// ---------------------------------------------------------------------------
// kernel timer: CUDA events around each launch on its own stream (the
// counterpart of the reference's profiling_in/out labels)
namespace {
struct ProfRec {
  const char *label;
  cudaEvent_t a, b;
};
std::mutex g_prof_mu;
bool g_prof_on = false;
std::vector<ProfRec> g_prof;
std::vector<cudaEvent_t> g_prof_pool;
size_t g_prof_used = 0;
cudaEvent_t prof_event() {
  if (g_prof_used == g_prof_pool.size()) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    g_prof_pool.push_back(e);
  }
  return g_prof_pool[g_prof_used++];
}
}  // namespace

ProfScope::ProfScope(const char *label, cudaStream_t st) : st_(st) {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  if (!g_prof_on || g_prof.size() >= (1u << 20)) return;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
    cudaGetLastError();
    return;  // no timing events inside a graph capture
  }
  ProfRec r{label, prof_event(), prof_event()};
  cudaEventRecord(r.a, st);
  g_prof.push_back(r);
  idx_ = long(g_prof.size()) - 1;
}
ProfScope::~ProfScope() {
  if (idx_ < 0) return;
  std::lock_guard<std::mutex> lk(g_prof_mu);
  cudaEventRecord(g_prof[idx_].b, st_);
}

// ---------------------------------------------------------------------------
// small device helpers
namespace {

__global__ void scatter_cells_kernel(const double *v, const int *cell_of_row, int n, double *vcell) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) vcell[cell_of_row[i]] = v[i];
}

// rho[r] (+)= the density of row r from the fused partials: the KB ket's row
// sums for covered rows (their final values), the pass's chunk sums elsewhere;
// fixed summation order.
__global__ void rho_finalize_kernel(const double *part, int chunks, const double *ket, int kxb, int nk,
                                    const int *kidx, int np, int acc, double *rho) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= np) return;
  double v = 0.0;
  const int k = kidx ? kidx[r] : -1;
  if (k >= 0)
    for (int b = 0; b < kxb; ++b) v += ket[(long long)b * nk + k];
  else
    for (int c = 0; c < chunks; ++c) v += part[(long long)c * np + r];
  rho[r] = acc ? rho[r] + v : v;
}

template <typename T>
__global__ void boundaries_kernel(T *psi, long long ld, int np, int nb, const int *per_inner, const T *phase,
                                  int periodic) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long n = (long long)nb * ld;
  if (i >= n) return;
  const int b = int(i / ld), s = int(i % ld);
  T *dst = psi + (long long)(np + b) * 2 * ld + 2 * s;
  if (!periodic) {
    dst[0] = T(0);
    dst[1] = T(0);
    return;
  }
  const T *src = psi + (long long)per_inner[b] * 2 * ld + 2 * s;
  if (phase) {
    const T pr = phase[2 * b], pi = phase[2 * b + 1];
    const T xr = src[0], xi = src[1];
    dst[0] = xr * pr - xi * pi;
    dst[1] = xr * pi + xi * pr;
  } else {
    dst[0] = src[0];
    dst[1] = src[1];
  }
}

template <typename T>
__global__ void copy_rows_kernel(const T *src, long long lds, T *dst, long long ldd, int nrows, int nst) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long n = (long long)nrows * nst;
  if (i >= n) return;
  const long long r = i / nst;
  const int s = int(i % nst);
  dst[r * 2 * ldd + 2 * s] = src[r * 2 * lds + 2 * s];
  dst[r * 2 * ldd + 2 * s + 1] = src[r * 2 * lds + 2 * s + 1];
}

}  // namespace

hpsi_status dev_alloc(void **p, size_t bytes) {
  if (bytes == 0) bytes = 16;
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    set_error(std::string("cudaMalloc(") + std::to_string(bytes) + "): " + cudaGetErrorString(e));
    return HPSI_ERR_NOMEM;
  }
  return HPSI_OK;
}

void dev_free(void *p) {
  if (p) cudaFree(p);
}

hpsi_status Workspace::ensure(size_t bytes) {
  if (bytes <= size) return HPSI_OK;
  dev_free(ptr);
  ptr = nullptr;
  size = 0;
  hpsi_status s = dev_alloc(&ptr, bytes);
  if (s == HPSI_OK) size = bytes;
  return s;
}

void Workspace::release() {
  dev_free(ptr);
  ptr = nullptr;
  size = 0;
}

// true if the pointer can be dereferenced by kernels on the current device
bool is_device_ptr(const void *p) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

hpsi_status check_batch(const hpsi_mesh *m, const hpsi_batch *b, int min_rows, const char *what) {
  if (!b || !b->ptr) {
    set_error(std::string(what) + ": null batch");
    return HPSI_ERR_ARG;
  }
  if (b->dtype != HPSI_C128 && b->dtype != HPSI_C64) {
    set_error(std::string(what) + ": unknown dtype");
    return HPSI_ERR_ARG;
  }
  if (b->nst < 1 || b->ld < b->nst) {
    set_error(std::string(what) + ": need 1 <= nst <= ld");
    return HPSI_ERR_ARG;
  }
  if (b->npts < min_rows) {
    set_error(std::string(what) + ": batch holds " + std::to_string(b->npts) + " points, need " +
              std::to_string(min_rows));
    return HPSI_ERR_ARG;
  }
  const size_t esz = b->dtype == HPSI_C128 ? 16 : 8;
  if ((reinterpret_cast<uintptr_t>(b->ptr) % 16) != 0 || (size_t(b->ld) * esz) % 16 != 0) {
    // the stencil gathers 16-byte pieces of each row
    if (!(b->dtype == HPSI_C64 && b->ld % 2 == 1 && b->ld == 1)) {
      set_error(std::string(what) + ": rows must start on 16-byte boundaries (ld * element size % 16 == 0)");
      return HPSI_ERR_ARG;
    }
  }
  (void)m;
  return HPSI_OK;
}

// state chunk width of the fused pass for a batch
int pass_sc(int dtype, long long ld) {
  const int maxsc = dtype == HPSI_C128 ? 4 : 8;
  for (int sc = maxsc; sc >= 1; sc >>= 1)
    if (ld % sc == 0) return sc;
  return 1;
}

// Shape of the cp.async pass (one complex state per thread, 16 x 16 tiles):
// a thread keeps RY rows of 9 complex running sums, FP64 2 rows, FP32 4.
PassShape legacy_shape(int dtype, long long ld) {
  const int sc = pass_sc(dtype, ld);
  return dtype == HPSI_C128 ? PassShape{sc, 16, 16, 2} : PassShape{sc, 16, 16, 4};
}

// Shape of the register-blocked pass (one real lane per thread, 16 x 8 tiles).
PassShape blk_shape(int dtype) {
  // measured on the R = 12 bohr sphere (128 states): FP64 2 x 2 cells of one
  // real lane (512 threads); FP32 2 x 2 cells of one complex state with
  // packed multiply-adds (512 threads)
  PassShape s = dtype == HPSI_C128 ? PassShape{blk_chunk_states<double>(), 16, 8, 2}
                                   : PassShape{blk_chunk_states<float>(), 16, 8, 2};
  s.blk = 1;
  s.rx = 2;
  s.cplx = dtype == HPSI_C128 ? 0 : 1;
  s.unroll = 9;  // planes per unrolled group of the z march (9: no rotation)
  return s;
}

// Register-blocked pass over half chunks (64 bytes: FP64 4 states, FP32 8),
// 16 x 8 tiles, 1 x 4 cells, 256 threads and two CTAs per SM: the default
// for widths that are a multiple of the half chunk but not of the chunk.
// Measured on the R = 12 sphere against the one-complex pass: FP32 8 / 24 /
// 40 states 0.144 / 0.302 / 0.414 -> 0.111 / 0.208 / 0.326 ms, FP64 4 / 12 /
// 20 states 0.133 / 0.284 / 0.384 -> 0.106 / 0.201 / 0.323 ms.
PassShape half_chunk_shape(int dtype) {
  PassShape s = blk_shape(dtype);
  s.sc /= 2;
  s.ty = 8;
  s.rx = 1;
  s.ry = 4;
  return s;
}

PassShape default_shape(int dtype, long long ld) {
  const PassShape b = blk_shape(dtype);
  PassShape s = ld % b.sc == 0         ? b
                : ld % (b.sc / 2) == 0 ? half_chunk_shape(dtype)
                                       : legacy_shape(dtype, ld);
  // experiment override: HPSI_PASS_SHAPE64 / HPSI_PASS_SHAPE32 = "sc,ry,zb,unroll,blk,rx,cplx,ty,tma,mb,mma"
  const char *env = std::getenv(dtype == HPSI_C128 ? "HPSI_PASS_SHAPE64" : "HPSI_PASS_SHAPE32");
  if (env) {
    int a = 0, b = 0, c = 0, u = 0, t = 0, x = 0, cx = -1, ty = 0, tm = 0, mb = 0, mm = 0;
    if (std::sscanf(env, "%d,%d,%d,%d,%d,%d,%d,%d,%d,%d,%d", &a, &b, &c, &u, &t, &x, &cx, &ty, &tm, &mb, &mm) >= 2 &&
        a > 0 &&
        ld % a == 0) {
      if (t) {
        s = blk_shape(dtype);  // chunk (128 or 64 bytes), block, element, z depth and group are taken
        if (a == s.sc / 2) {
          s.sc = a;  // 64-byte chunks ride 16 x 16 tiles unless ty = 8 is given
          s.ty = ty == 8 ? 8 : 16;
        }
        if (u == 1 || u == 3 || u == 9) s.unroll = u;
        if (x > 0) s.rx = x;
        if (b > 0) s.ry = b;
        if (cx >= 0) s.cplx = cx;
        s.tma = tm ? 1 : 0;
        s.mb = mb ? 1 : 0;
        s.mma = mm ? 1 : 0;
      } else {
        s = legacy_shape(dtype, ld);
        s.sc = a;
        s.ry = b;
      }
      s.zb = c;
    }
  }
  return s;
}

}  // namespace hpsi

using namespace hpsi;

// ===========================================================================
extern "C" {

const char *hpsi_last_error_string(void) { return t_last_error.c_str(); }
int64_t hpsi_kernel_launch_count(void) { return g_launches.load(); }
const char *hpsi_version(void) { return "hpsi 0.1 (sm_100a)"; }

hpsi_status hpsi_profile_enable(int32_t on) {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  g_prof.clear();
  g_prof_used = 0;
  g_prof_on = on != 0;
  return HPSI_OK;
}

hpsi_status hpsi_profile_query(const char *label, int64_t *launches, double *total_ms) {
  if (!label || !launches || !total_ms) return HPSI_ERR_ARG;
  std::lock_guard<std::mutex> lk(g_prof_mu);
  *launches = 0;
  *total_ms = 0.0;
  for (auto &r : g_prof) {
    if (std::strcmp(r.label, label) != 0) continue;
    cudaError_t e = cudaEventSynchronize(r.b);
    if (e != cudaSuccess) {
      set_error(std::string("hpsi_profile_query: ") + cudaGetErrorString(e));
      return HPSI_ERR_CUDA;
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, r.a, r.b);
    *launches += 1;
    *total_ms += ms;
  }
  return HPSI_OK;
}

hpsi_status hpsi_mesh_create(const hpsi_mesh_desc *d, hpsi_mesh **out) {
  if (!d || !out || !d->lxyz || d->np < 1 || d->np_part < d->np) {
    set_error("hpsi_mesh_create: bad descriptor");
    return HPSI_ERR_ARG;
  }
  if (d->order < 1 || d->order > 4) {
    set_error("hpsi_mesh_create: stencil order must be 1..4");
    return HPSI_ERR_UNSUPPORTED;
  }
  if (d->periodic && !d->per_inner && d->np_part > d->np) {
    set_error("hpsi_mesh_create: periodic mesh without per_inner");
    return HPSI_ERR_ARG;
  }
  const int np = d->np, npp = d->np_part, HAL = 4;
  int lo[3], hi[3];
  for (int a = 0; a < 3; ++a) {
    lo[a] = d->lxyz[a];
    hi[a] = d->lxyz[a];
  }
  for (int i = 0; i < np; ++i)
    for (int a = 0; a < 3; ++a) {
      lo[a] = std::min(lo[a], d->lxyz[3 * i + a]);
      hi[a] = std::max(hi[a], d->lxyz[3 * i + a]);
    }
  CellBox B;
  B.halo = HAL;
  B.nxo = hi[0] - lo[0] + 1;
  B.nyo = hi[1] - lo[1] + 1;
  B.nzo = hi[2] - lo[2] + 1;
  B.NX = (B.nxo + 31) / 32 * 32 + 2 * HAL;
  B.NY = (B.nyo + 31) / 32 * 32 + 2 * HAL;
  B.NZ = B.nzo + 2 * HAL;
  for (int a = 0; a < 3; ++a) {
    B.lo[a] = lo[a] - HAL;
    B.h[a] = d->spacing[a];
  }
  const long long ncell = (long long)B.NX * B.NY * B.NZ;
  if (ncell > (1LL << 31) - 1 || (long long)npp * 4096 > (1LL << 62)) {
    set_error("hpsi_mesh_create: mesh too large");
    return HPSI_ERR_UNSUPPORTED;
  }
  std::vector<int> cell_row(ncell, -1), cell_of_row(npp);
  for (int i = 0; i < npp; ++i) {
    const int x = d->lxyz[3 * i] - B.lo[0], y = d->lxyz[3 * i + 1] - B.lo[1], z = d->lxyz[3 * i + 2] - B.lo[2];
    if (x < 0 || y < 0 || z < 0 || x >= B.NX || y >= B.NY || z >= B.NZ) {
      set_error("hpsi_mesh_create: boundary point " + std::to_string(i) +
                " is farther than 4 cells from the inner points");
      return HPSI_ERR_INDEX;
    }
    const long long c = ((long long)z * B.NY + y) * B.NX + x;
    if (cell_row[c] != -1) {
      set_error("hpsi_mesh_create: duplicate point " + std::to_string(i));
      return HPSI_ERR_INDEX;
    }
    cell_row[c] = i;
    cell_of_row[i] = int(c);
  }
  // every star neighbour (half-width = order) of an inner point must exist
  const int ord = d->order;
  for (int i = 0; i < np; ++i) {
    const long long c = cell_of_row[i];
    const long long strides[3] = {1, B.NX, (long long)B.NX * B.NY};
    for (int a = 0; a < 3; ++a)
      for (int s = -ord; s <= ord; ++s) {
        if (!s) continue;
        if (cell_row[c + s * strides[a]] < 0) {
          set_error("hpsi_mesh_create: stencil of inner point " + std::to_string(i) + " leaves the mesh");
          return HPSI_ERR_INDEX;
        }
      }
  }
  std::vector<int> src_zero(ncell), src_per;
  for (long long c = 0; c < ncell; ++c) src_zero[c] = (cell_row[c] >= 0 && cell_row[c] < np) ? cell_row[c] : -1;
  std::vector<int> per;
  if (d->periodic) {
    per.assign(d->per_inner, d->per_inner + (npp - np));
    for (int b = 0; b < npp - np; ++b)
      if (per[b] < 0 || per[b] >= np) {
        set_error("hpsi_mesh_create: per_inner[" + std::to_string(b) + "] is not an inner point");
        return HPSI_ERR_INDEX;
      }
    src_per = src_zero;
    for (int b = 0; b < npp - np; ++b) src_per[cell_of_row[np + b]] = per[b];
  }
  hpsi_mesh *m = new hpsi_mesh();
  m->tiles_x = (B.nxo + PASS_TILE - 1) / PASS_TILE;
  m->tiles_y = (B.nyo + PASS_TILE - 1) / PASS_TILE;
  m->tile_z.assign(size_t(m->tiles_x) * m->tiles_y, make_int2(1 << 30, -1));
  for (int i = 0; i < np; ++i) {
    const int c = cell_of_row[i];
    const int x = c % B.NX, y = (c / B.NX) % B.NY, z = c / (B.NX * B.NY);
    int2 &t = m->tile_z[size_t((y - HAL) / PASS_TILE) * m->tiles_x + (x - HAL) / PASS_TILE];
    t.x = std::min(t.x, z);
    t.y = std::max(t.y, z);
  }
  for (auto &t : m->tile_z)
    if (t.y >= 0) m->column_planes += t.y - t.x + 1;
  m->tiles_y8 = 2 * m->tiles_y;
  m->tile_z8.assign(size_t(m->tiles_x) * m->tiles_y8, make_int2(1 << 30, -1));
  std::vector<int2> col_z(size_t(B.NX) * B.NY, make_int2(1 << 30, -(1 << 30)));
  for (int i = 0; i < np; ++i) {
    const int c = cell_of_row[i];
    const int x = c % B.NX, y = (c / B.NX) % B.NY, z = c / (B.NX * B.NY);
    int2 &t = m->tile_z8[size_t((y - HAL) / 8) * m->tiles_x + (x - HAL) / PASS_TILE];
    t.x = std::min(t.x, z);
    t.y = std::max(t.y, z);
    int2 &cz = col_z[size_t(y) * B.NX + x];
    cz.x = std::min(cz.x, z);
    cz.y = std::max(cz.y, z);
  }
  m->np = np;
  m->np_part = npp;
  m->order = ord;
  m->periodic = d->periodic ? 1 : 0;
  m->box = B;
  m->per_inner_h = per;
  m->cell_of_row_h = cell_of_row;
  m->cell_row_h = cell_row;
  cudaGetDevice(&m->device);
  cudaDeviceGetAttribute(&m->num_sms, cudaDevAttrMultiProcessorCount, m->device);
  hpsi_status s = HPSI_OK;
  auto up = [&](int **dp, const std::vector<int> &h) {
    if (s != HPSI_OK) return;
    s = dev_alloc(reinterpret_cast<void **>(dp), h.size() * sizeof(int));
    if (s == HPSI_OK && !h.empty()) {
      cudaError_t e = cudaMemcpy(*dp, h.data(), h.size() * sizeof(int), cudaMemcpyHostToDevice);
      if (e != cudaSuccess) {
        set_error(std::string("hpsi_mesh_create: ") + cudaGetErrorString(e));
        s = HPSI_ERR_CUDA;
      }
    }
  };
  up(&m->d_cell_row, cell_row);
  up(&m->d_src_raw, cell_row);
  if (s == HPSI_OK) {
    s = dev_alloc(reinterpret_cast<void **>(&m->d_col_z), col_z.size() * sizeof(int2));
    if (s == HPSI_OK) {
      cudaError_t e = cudaMemcpy(m->d_col_z, col_z.data(), col_z.size() * sizeof(int2), cudaMemcpyHostToDevice);
      if (e != cudaSuccess) {
        set_error(cudaGetErrorString(e));
        s = HPSI_ERR_CUDA;
      }
    }
  }
  up(&m->d_src_zero, src_zero);
  up(&m->d_cell_of_row, cell_of_row);
  if (m->periodic) {
    up(&m->d_src_per, src_per);
    up(&m->d_per_inner, per);
  }
  if (s != HPSI_OK) {
    hpsi_mesh_destroy(m);
    return s;
  }
  *out = m;
  return HPSI_OK;
}

hpsi_status hpsi_mesh_destroy(hpsi_mesh *m) {
  if (!m) return HPSI_OK;
  dev_free(m->d_cell_row);
  dev_free(m->d_src_raw);
  dev_free(m->d_src_zero);
  dev_free(m->d_src_per);
  dev_free(m->d_per_inner);
  dev_free(m->d_cell_of_row);
  dev_free(m->d_col_z);
  m->scratch.release();
  m->scratch2.release();
  for (auto &kv : m->items) dev_free(kv.second.first);
  for (auto &kv : m->items_part) dev_free(kv.second.first);
  for (auto &kv : m->seg_masks) dev_free(kv.second);
  m->stage_in.release();
  m->stage_out.release();
  delete m;
  return HPSI_OK;
}

hpsi_status hpsi_mesh_info(const hpsi_mesh *m, int32_t dims[6]) {
  if (!m || !dims) return HPSI_ERR_ARG;
  dims[0] = m->box.NX;
  dims[1] = m->box.NY;
  dims[2] = m->box.NZ;
  dims[3] = m->box.nxo;
  dims[4] = m->box.nyo;
  dims[5] = m->box.nzo;
  return HPSI_OK;
}

// ---------------------------------------------------------------------------
hpsi_status hpsi_hamiltonian_create(hpsi_mesh *mesh, hpsi_hamiltonian **out) {
  if (!mesh || !out) return HPSI_ERR_ARG;
  hpsi_hamiltonian *h = new hpsi_hamiltonian();
  h->mesh = mesh;
  // experiment override: HPSI_BRA_OVERLAP=0 runs the KB bra on the caller's
  // stream before the pass
  if (const char *e = std::getenv("HPSI_BRA_OVERLAP")) h->overlap_bra = std::atoi(e) != 0;
  if (const char *e = std::getenv("HPSI_PASS_PRIORITY")) h->prio_pass = std::atoi(e) != 0;
  // experiment override: HPSI_FUSED_DENSITY=1 fuses the density of
  // hpsi_taylor_step_density into the last pass
  if (const char *e = std::getenv("HPSI_FUSED_DENSITY")) h->fuse_density = std::atoi(e) != 0;
  *out = h;
  return HPSI_OK;
}

hpsi_status hpsi_hamiltonian_destroy(hpsi_hamiltonian *h) {
  if (!h) return HPSI_OK;
  dev_free(h->d_vcell);
  dev_free(h->d_phase);
  dev_free(h->d_phase_f);
  dev_free(h->d_src_phase);
  h->proj_free();
  for (auto &w : h->u) w.release();
  h->projbuf.release();
  h->bra_partial.release();
  h->obsbuf.release();
  h->ketobs.release();
  h->tdbuf.release();
  h->adjbuf.release();
  h->lzbuf.release();
  h->vstage.release();
  h->adjstep.release();
  h->vjpbuf.release();
  h->rhobuf.release();
  dev_free(h->d_err);
  h->lzsmall.release();
  if (h->bra_stream) cudaStreamDestroy(h->bra_stream);
  if (h->pass_stream) cudaStreamDestroy(h->pass_stream);
  if (h->pass_join) cudaEventDestroy(h->pass_join);
  if (h->bra_fork) cudaEventDestroy(h->bra_fork);
  if (h->bra_join) cudaEventDestroy(h->bra_join);
  if (h->capture_stream) cudaStreamDestroy(h->capture_stream);
  if (h->capture_event) cudaEventDestroy(h->capture_event);
  if (h->xfer_in) cudaStreamDestroy(h->xfer_in);
  if (h->xfer_out) cudaStreamDestroy(h->xfer_out);
  for (auto &e : h->xev)
    if (e) cudaEventDestroy(e);
  h->slab_in.release();
  h->slab_out.release();
  h->small.release();
  delete h;
  return HPSI_OK;
}

hpsi_status hpsi_hamiltonian::ensure_bra_stream() {
  if (bra_stream) return HPSI_OK;
  HPSI_TRY_CUDA(cudaStreamCreateWithFlags(&bra_stream, cudaStreamNonBlocking));
  HPSI_TRY_CUDA(cudaEventCreateWithFlags(&bra_fork, cudaEventDisableTiming));
  HPSI_TRY_CUDA(cudaEventCreateWithFlags(&bra_join, cudaEventDisableTiming));
  int least = 0, greatest = 0;
  HPSI_TRY_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
  HPSI_TRY_CUDA(cudaStreamCreateWithPriority(&pass_stream, cudaStreamNonBlocking, greatest));
  HPSI_TRY_CUDA(cudaEventCreateWithFlags(&pass_join, cudaEventDisableTiming));
  return HPSI_OK;
}

void hpsi_hamiltonian::proj_free() {
  dev_free(d_mat);
  dev_free(d_proj_row);
  dev_free(d_map);
  dev_free(d_pt);
  dev_free(d_pt_f);
  dev_free(d_scal);
  dev_free(d_scal_f);
  dev_free(d_krows);
  dev_free(d_kidx);
  d_kidx = nullptr;
  dev_free(d_kptr);
  dev_free(d_kb_ent);
  dev_free(d_kb_phase);
  dev_free(d_kb_phase_f);
  d_kb_phase = nullptr;
  d_kb_phase_f = nullptr;
  kb_npts = 0;
  kb_npoints_h.clear();
  d_mat = nullptr;
  d_proj_row = d_map = d_krows = d_kptr = nullptr;
  nk = 0;
  min_npoints = 0;
  d_pt = d_scal = nullptr;
  d_pt_f = d_scal_f = nullptr;
  d_kb_ent = nullptr;
  nmat = 0;
  nprojections = 0;
  max_nproj = 0;
}

hpsi_status hpsi_hamiltonian_set_kinetic(hpsi_hamiltonian *h, int32_t W, const int32_t *points, const double *w,
                                         double factor) {
  if (!h || !points || !w || W < 1) return HPSI_ERR_ARG;
  for (int k = 0; k < 9; ++k) h->wx[k] = h->wy[k] = h->wz[k] = 0.0;
  int ncenter = 0;
  for (int j = 0; j < W; ++j) {
    const int dx = points[3 * j], dy = points[3 * j + 1], dz = points[3 * j + 2];
    const int nz = (dx != 0) + (dy != 0) + (dz != 0);
    if (nz > 1 || std::abs(dx) > 4 || std::abs(dy) > 4 || std::abs(dz) > 4 ||
        std::max({std::abs(dx), std::abs(dy), std::abs(dz)}) > h->mesh->order) {
      set_error("hpsi_hamiltonian_set_kinetic: only star stencils within the mesh order are supported");
      return HPSI_ERR_UNSUPPORTED;
    }
    const double wf = w[j] * factor;  // the reference multiplies op%w by the factor (nl_operator_inc.F90:72-80)
    if (nz == 0) {
      h->wx[4] += wf;
      ++ncenter;
    } else if (dx)
      h->wx[dx + 4] += wf;
    else if (dy)
      h->wy[dy + 4] += wf;
    else
      h->wz[dz + 4] += wf;
  }
  if (ncenter != 1) {
    set_error("hpsi_hamiltonian_set_kinetic: the stencil must contain the centre exactly once");
    return HPSI_ERR_ARG;
  }
  h->have_kinetic = true;
  return HPSI_OK;
}

// Writes v (np doubles, host or device) into the cell array of the potential
// on `st`.  The cell array and, for host input, the staging buffer are
// allocated on the first call and reused afterwards.
static hpsi_status vloc_write(hpsi_hamiltonian *h, const double *v, cudaStream_t st, const char *who) {
  hpsi_mesh *m = h->mesh;
  const long long ncell = (long long)m->box.NX * m->box.NY * m->box.NZ;
  const bool dev_in = is_device_ptr(v);
  if (!dev_in)
    for (int i = 0; i < m->np; ++i)
      if (!std::isfinite(v[i])) {
        set_error(std::string(who) + ": non-finite potential at point " + std::to_string(i));
        return HPSI_ERR_NONFINITE;
      }
  if (!h->d_vcell) {
    hpsi_status s = dev_alloc(reinterpret_cast<void **>(&h->d_vcell), ncell * sizeof(double));
    if (s) return s;
    // cells that hold no inner point stay zero from here on
    HPSI_TRY_CUDA(cudaMemsetAsync(h->d_vcell, 0, ncell * sizeof(double), st));
  }
  const double *src = v;
  if (!dev_in) {
    hpsi_status s = h->vstage.ensure(size_t(m->np) * sizeof(double));
    if (s) return s;
    HPSI_TRY_CUDA(cudaMemcpyAsync(h->vstage.ptr, v, size_t(m->np) * sizeof(double), cudaMemcpyHostToDevice, st));
    src = static_cast<const double *>(h->vstage.ptr);
  }
  scatter_cells_kernel<<<(m->np + 255) / 256, 256, 0, st>>>(src, m->d_cell_of_row, m->np, h->d_vcell);
  g_launches++;
  HPSI_CHECK_LAUNCH();
  return HPSI_OK;
}

hpsi_status hpsi_hamiltonian_set_vloc(hpsi_hamiltonian *h, const double *v) {
  if (!h) return HPSI_ERR_ARG;
  if (!v) {
    dev_free(h->d_vcell);
    h->d_vcell = nullptr;
    return HPSI_OK;
  }
  hpsi_status s = vloc_write(h, v, nullptr, "hpsi_hamiltonian_set_vloc");
  if (s) return s;
  // the set-up call returns with the potential in place (legacy stream only)
  cudaError_t e = cudaStreamSynchronize(nullptr);
  if (e != cudaSuccess) {
    set_error(std::string("hpsi_hamiltonian_set_vloc: ") + cudaGetErrorString(e));
    return HPSI_ERR_CUDA;
  }
  return HPSI_OK;
}

hpsi_status hpsi_hamiltonian_update_vloc(hpsi_hamiltonian *h, const double *v, void *stream) {
  if (!h || !v) {
    set_error("hpsi_hamiltonian_update_vloc: null argument");
    return HPSI_ERR_ARG;
  }
  return vloc_write(h, v, static_cast<cudaStream_t>(stream), "hpsi_hamiltonian_update_vloc");
}

hpsi_status hpsi_hamiltonian_set_field(hpsi_hamiltonian *h, const double pol[3], double amplitude) {
  if (!h || !pol) return HPSI_ERR_ARG;
  for (int a = 0; a < 3; ++a) {
    h->pol[a] = pol[a];
    h->fld[a] = pol[a] * amplitude;
  }
  h->have_pol = true;
  return HPSI_OK;
}

hpsi_status hpsi_hamiltonian_set_phase_corr(hpsi_hamiltonian *h, const double *pc) {
  if (!h) return HPSI_ERR_ARG;
  hpsi_mesh *m = h->mesh;
  dev_free(h->d_phase);
  dev_free(h->d_phase_f);
  dev_free(h->d_src_phase);
  h->d_phase = nullptr;
  h->d_phase_f = nullptr;
  h->d_src_phase = nullptr;
  if (!pc) return HPSI_OK;
  if (!m->periodic) {
    set_error("hpsi_hamiltonian_set_phase_corr: mesh is not periodic");
    return HPSI_ERR_STATE;
  }
  const int nb = m->np_part - m->np;
  std::vector<float> pf(2 * size_t(nb));
  for (size_t i = 0; i < pf.size(); ++i) pf[i] = float(pc[i]);
  // encoded load map: boundary cell -> -(b + 2)
  const long long ncell = (long long)m->box.NX * m->box.NY * m->box.NZ;
  std::vector<int> enc(ncell);
  HPSI_TRY_CUDA(cudaMemcpy(enc.data(), m->d_src_zero, ncell * sizeof(int), cudaMemcpyDeviceToHost));
  for (int b = 0; b < nb; ++b) enc[m->cell_of_row_h[m->np + b]] = -(b + 2);
  hpsi_status s = dev_alloc(reinterpret_cast<void **>(&h->d_phase), 2 * size_t(nb) * sizeof(double));
  if (!s) s = dev_alloc(reinterpret_cast<void **>(&h->d_phase_f), 2 * size_t(nb) * sizeof(float));
  if (!s) s = dev_alloc(reinterpret_cast<void **>(&h->d_src_phase), ncell * sizeof(int));
  if (s) return s;
  HPSI_TRY_CUDA(cudaMemcpy(h->d_phase, pc, 2 * size_t(nb) * sizeof(double), cudaMemcpyHostToDevice));
  HPSI_TRY_CUDA(cudaMemcpy(h->d_phase_f, pf.data(), pf.size() * sizeof(float), cudaMemcpyHostToDevice));
  HPSI_TRY_CUDA(cudaMemcpy(h->d_src_phase, enc.data(), ncell * sizeof(int), cudaMemcpyHostToDevice));
  return HPSI_OK;
}

hpsi_status hpsi_hamiltonian_set_projectors(hpsi_hamiltonian *h, int32_t nmat, const int32_t *npoints,
                                            const int32_t *nprojs, const int32_t *map, const double *matrices,
                                            const double *scal) {
  if (!h || nmat < 0) return HPSI_ERR_ARG;
  h->proj_free();
  if (nmat == 0) return HPSI_OK;
  if (!npoints || !nprojs || !map || !matrices || !scal) return HPSI_ERR_ARG;
  hpsi_mesh *m = h->mesh;
  std::vector<int4> mat(nmat);
  std::vector<int> prow(nmat);
  long long npts_tot = 0, nval = 0;
  int nproj_tot = 0, maxp = 0;
  for (int i = 0; i < nmat; ++i) {
    if (npoints[i] < 0 || nprojs[i] < 1) {
      set_error("hpsi_hamiltonian_set_projectors: bad matrix size");
      return HPSI_ERR_ARG;
    }
    mat[i] = make_int4(npoints[i], nprojs[i], int(npts_tot), int(nval));
    prow[i] = nproj_tot;
    npts_tot += npoints[i];
    nval += (long long)npoints[i] * nprojs[i];
    nproj_tot += nprojs[i];
    maxp = std::max(maxp, int(nprojs[i]));
  }
  if (nval > (1LL << 31) - 1) return HPSI_ERR_UNSUPPORTED;
  std::vector<double> pt(nval);
  std::vector<float> ptf(nval), scf(nproj_tot);
  std::vector<int> cnt(m->np + 1, 0);
  for (int i = 0; i < nmat; ++i) {
    const int n = npoints[i], q = nprojs[i];
    const double *src = matrices + mat[i].w;
    for (int k = 0; k < n; ++k) {
      const int row = map[mat[i].z + k];
      if (row < 0 || row >= m->np) {
        set_error("hpsi_hamiltonian_set_projectors: map entry " + std::to_string(mat[i].z + k) +
                  " is not an inner point");
        return HPSI_ERR_INDEX;
      }
      cnt[row + 1]++;
      for (int j = 0; j < q; ++j) {
        pt[mat[i].w + (long long)k * q + j] = src[(long long)j * n + k];
        ptf[mat[i].w + (long long)k * q + j] = float(src[(long long)j * n + k]);
      }
    }
  }
  for (int i = 0; i < nproj_tot; ++i) scf[i] = float(scal[i]);
  for (int r = 0; r < m->np; ++r) cnt[r + 1] += cnt[r];
  std::vector<int4> ent(npts_tot);
  std::vector<int> fill(cnt.begin(), cnt.end() - 1);
  for (int i = 0; i < nmat; ++i)
    for (int k = 0; k < npoints[i]; ++k) {
      const int row = map[mat[i].z + k];
      ent[fill[row]++] = make_int4(mat[i].w + k * nprojs[i], prow[i], nprojs[i], mat[i].z + k);
    }
  // compress to the covered rows (entries stay in matrix order per row)
  std::vector<int> krows, kptr(1, 0);
  for (int r = 0; r < m->np; ++r)
    if (cnt[r + 1] > cnt[r]) {
      krows.push_back(r);
      kptr.push_back(cnt[r + 1]);
    }
  int minp = 1 << 30;
  for (int i = 0; i < nmat; ++i) minp = std::min(minp, int(npoints[i]));
  hpsi_status s = HPSI_OK;
  auto up = [&](void **dp, const void *src, size_t bytes) {
    if (s) return;
    s = dev_alloc(dp, bytes);
    if (!s && bytes) {
      cudaError_t e = cudaMemcpy(*dp, src, bytes, cudaMemcpyHostToDevice);
      if (e != cudaSuccess) {
        set_error(cudaGetErrorString(e));
        s = HPSI_ERR_CUDA;
      }
    }
  };
  up(reinterpret_cast<void **>(&h->d_mat), mat.data(), mat.size() * sizeof(int4));
  up(reinterpret_cast<void **>(&h->d_proj_row), prow.data(), prow.size() * sizeof(int));
  up(reinterpret_cast<void **>(&h->d_map), map, size_t(npts_tot) * sizeof(int));
  up(reinterpret_cast<void **>(&h->d_pt), pt.data(), pt.size() * sizeof(double));
  up(reinterpret_cast<void **>(&h->d_pt_f), ptf.data(), ptf.size() * sizeof(float));
  up(reinterpret_cast<void **>(&h->d_scal), scal, size_t(nproj_tot) * sizeof(double));
  up(reinterpret_cast<void **>(&h->d_scal_f), scf.data(), scf.size() * sizeof(float));
  up(reinterpret_cast<void **>(&h->d_krows), krows.data(), krows.size() * sizeof(int));
  {
    std::vector<int> kidx(m->np, -1);
    for (size_t i = 0; i < krows.size(); ++i) kidx[krows[i]] = int(i);
    up(reinterpret_cast<void **>(&h->d_kidx), kidx.data(), kidx.size() * sizeof(int));
  }
  up(reinterpret_cast<void **>(&h->d_kptr), kptr.data(), kptr.size() * sizeof(int));
  up(reinterpret_cast<void **>(&h->d_kb_ent), ent.data(), ent.size() * sizeof(int4));
  if (s) {
    h->proj_free();
    return s;
  }
  h->nmat = nmat;
  h->nprojections = nproj_tot;
  h->max_nproj = maxp;
  h->nk = int(krows.size());
  h->min_npoints = minp;
  h->kb_npts = npts_tot;
  h->kb_npoints_h.assign(npoints, npoints + nmat);
  return HPSI_OK;
}

hpsi_status hpsi_hamiltonian_set_projector_phases(hpsi_hamiltonian *h, const double *phases, int32_t ld_points) {
  if (!h) return HPSI_ERR_ARG;
  dev_free(h->d_kb_phase);
  dev_free(h->d_kb_phase_f);
  h->d_kb_phase = nullptr;
  h->d_kb_phase_f = nullptr;
  if (!phases) return HPSI_OK;
  if (h->nmat == 0) {
    set_error("hpsi_hamiltonian_set_projector_phases: no projectors set");
    return HPSI_ERR_STATE;
  }
  int maxn = 0;
  for (int n : h->kb_npoints_h) maxn = std::max(maxn, n);
  if (ld_points != 0 && ld_points < maxn) {
    set_error("hpsi_hamiltonian_set_projector_phases: ld_points " + std::to_string(ld_points) +
              " is below the largest sphere (" + std::to_string(maxn) + " points)");
    return HPSI_ERR_ARG;
  }
  // packed copy in the order of the map: matrix m's points start at
  // sum(npoints[0..m-1]) in the packed form, at m * ld_points in the padded one
  const size_t n = 2 * size_t(h->kb_npts);
  std::vector<double> pd(n);
  std::vector<float> pf(n);
  size_t o = 0;
  for (size_t m = 0; m < h->kb_npoints_h.size(); ++m) {
    const size_t src0 = ld_points ? 2 * m * size_t(ld_points) : o;
    for (int k = 0; k < h->kb_npoints_h[m]; ++k)
      for (int c = 0; c < 2; ++c) {
        const double x = phases[src0 + 2 * size_t(k) + c];
        if (!std::isfinite(x)) {
          set_error("hpsi_hamiltonian_set_projector_phases: non-finite phase of matrix " + std::to_string(m) +
                    ", point " + std::to_string(k));
          return HPSI_ERR_NONFINITE;
        }
        pd[o + 2 * size_t(k) + c] = x;
        pf[o + 2 * size_t(k) + c] = float(x);
      }
    o += 2 * size_t(h->kb_npoints_h[m]);
  }
  hpsi_status s = dev_alloc(reinterpret_cast<void **>(&h->d_kb_phase), n * sizeof(double));
  if (!s) s = dev_alloc(reinterpret_cast<void **>(&h->d_kb_phase_f), n * sizeof(float));
  if (s) return s;
  HPSI_TRY_CUDA(cudaMemcpy(h->d_kb_phase, pd.data(), n * sizeof(double), cudaMemcpyHostToDevice));
  HPSI_TRY_CUDA(cudaMemcpy(h->d_kb_phase_f, pf.data(), n * sizeof(float), cudaMemcpyHostToDevice));
  return HPSI_OK;
}

}  // extern "C"

// ===========================================================================
namespace hpsi {

// z block depth of a pass: the largest depth that still gives about four
// waves of CTAs (each block re-reads a 4-plane halo above and below).
// ty: tile height of the pass (16, or 8 for the blocked pass).
int choose_zb(const hpsi_mesh *m, int chunks, int ty) {
  const long long want = 4LL * m->num_sms;
  const int cands[] = {1 << 20, 96, 64, 48, 32, 24, 16};
  const auto &tz = ty == 8 ? m->tile_z8 : m->tile_z;
  for (int zb : cands) {
    long long n = 0;
    for (auto &t : tz)
      if (t.y >= 0) n += (t.y - t.x + zb) / zb;
    if (n * chunks >= want) return zb;
  }
  return 16;
}
int choose_zb(const hpsi_mesh *m, int chunks) { return choose_zb(m, chunks, 16); }

// z block depth of a single-system pass over 16 x 8 tiles (the blocked pass,
// ctas_per_sm resident CTAs per SM): the candidate with the shortest
// simulated makespan.  The
// work units, in launch order (z band, then column-major over the tiles; the
// state chunks of a unit consecutive), go one after another to the CTA slot that
// frees first, as the block scheduler hands them out; a unit costs its output
// planes + 8 halo planes + 4 (prologue).  Deeper blocks read fewer halo planes,
// shallower ones balance the tail: on the R = 12 sphere (108 tile columns) the
// choice is within 0.2 % of the best measured depth for 1 to 16 chunks, where
// a fixed four-wave target was up to 9.5 % slower with one or two chunks.
int choose_zb_single(const hpsi_mesh *m, int chunks, int ctas_per_sm) {
  const int key = 4 * chunks + ctas_per_sm;
  auto it = m->zb_single.find(key);
  if (it != m->zb_single.end()) return it->second;
  const int cands[] = {1 << 20, 96, 64, 48, 32, 24, 16};
  int best = 16;
  double best_t = 1e300;
  const int slots = std::max(1, m->num_sms * ctas_per_sm);
  for (int zb : cands) {
    std::vector<int4> u;  // {band, tile x, tile y, planes}
    for (int by = 0; by < m->tiles_y8; ++by)
      for (int bx = 0; bx < m->tiles_x; ++bx) {
        const int2 t = m->tile_z8[size_t(by) * m->tiles_x + bx];
        if (t.y < 0) continue;
        for (int z = t.x; z <= t.y; z += zb) u.push_back(make_int4(z / zb, bx, by, std::min(zb, t.y + 1 - z)));
      }
    std::stable_sort(u.begin(), u.end(), [](const int4 &a, const int4 &b) {
      if (a.x != b.x) return a.x < b.x;
      if (a.y != b.y) return a.y < b.y;
      return a.z < b.z;
    });
    std::priority_queue<double, std::vector<double>, std::greater<double>> free_at;
    for (int i = 0; i < slots; ++i) free_at.push(0.0);
    double end = 0.0;
    for (const int4 &w : u)
      for (int c = 0; c < chunks; ++c) {
        const double t = free_at.top() + double(w.w + 8 + 4);
        free_at.pop();
        free_at.push(t);
        end = std::max(end, t);
      }
    if (end < best_t) {
      best_t = end;
      best = zb;
    }
  }
  m->zb_single[key] = best;
  return best;
}

// z block depth of a single-system pass of a shape: the simulated choice for
// the blocked shapes over 16 x 8 tiles (128-byte chunks: one CTA per SM,
// 64-byte chunks with 1 x 4 cells: two), the four-wave target otherwise
int pass_zb(const hpsi_mesh *m, const PassShape &sh, int dtype, int chunks) {
  const int ty = sh.blk ? sh.ty : 16;
  const PassShape b = blk_shape(dtype);
  if (sh.blk && ty == 8 && sh.sc == b.sc) return choose_zb_single(m, chunks, 1);
  if (sh.blk && ty == 8 && sh.sc == b.sc / 2 && sh.rx == 1 && sh.ry == 4) return choose_zb_single(m, chunks, 2);
  return choose_zb(m, chunks, ty);
}

// Work list {tile x, tile y, first plane, end plane} for a z block depth and
// tile height (16: 16 x 16 tiles, 8: 16 x 8 tiles, tile y in 8-row units).
hpsi_status mesh_items(hpsi_mesh *m, int zb, int ty, const int4 **items, int *nitems) {
  const int key = 2 * zb + (ty == 8 ? 1 : 0);
  auto it = m->items.find(key);
  if (it == m->items.end()) {
    std::vector<int4> v;
    const int tyn = ty == 8 ? m->tiles_y8 : m->tiles_y;
    const auto &tz = ty == 8 ? m->tile_z8 : m->tile_z;
    for (int by = 0; by < tyn; ++by)
      for (int bx = 0; bx < m->tiles_x; ++bx) {
        const int2 t = tz[size_t(by) * m->tiles_x + bx];
        if (t.y < 0) continue;
        for (int z = t.x; z <= t.y; z += zb) v.push_back(make_int4(bx, by, z, std::min(z + zb, t.y + 1)));
      }
    // launch order: by z band, then column-major over the tiles (tile y
    // fastest), so that the CTAs in flight together are spatial neighbours and
    // share their halo rows in L2.  A tile's y halo (4 rows above and below,
    // 128 cells) is twice its x halo (64 cells): with y fastest the y
    // neighbours run together.  On the R = 12 sphere (128 states, FP64) the
    // pass read 3.29 GB from DRAM instead of 4.09 GB in raster order and ran
    // 0.5 % faster (FP32 1.1 %); strips of 2-6 tile columns and Morton order
    // measured slower.
    std::stable_sort(v.begin(), v.end(), [zb](const int4 &a, const int4 &b) {
      const int za = a.z / zb, zbb = b.z / zb;
      if (za != zbb) return za < zbb;
      if (a.x != b.x) return a.x < b.x;
      return a.y < b.y;
    });
    int4 *d = nullptr;
    hpsi_status s = dev_alloc(reinterpret_cast<void **>(&d), std::max<size_t>(1, v.size()) * sizeof(int4));
    if (s) return s;
    if (!v.empty()) HPSI_TRY_CUDA(cudaMemcpy(d, v.data(), v.size() * sizeof(int4), cudaMemcpyHostToDevice));
    it = m->items.emplace(key, std::make_pair(d, int(v.size()))).first;
  }
  *items = it->second.first;
  *nitems = it->second.second;
  return HPSI_OK;
}
hpsi_status mesh_items(hpsi_mesh *m, int zb, const int4 **items, int *nitems) {
  return mesh_items(m, zb, 16, items, nitems);
}

// Work list of one part of a domain-parallel mesh (part 1: output planes of a
// tile column whose stencil reads no ghost row; part 2: the others), the
// split the reference makes between op%inner and op%outer
// (src/grid/nl_operator.F90:458-514) so that the inner points run while the
// ghost rows are in flight (src/grid/derivatives_inc.F90:82-102).  A plane of
// a tile column is marked ghost-reading, conservatively, when a ghost cell lies
// in the tile's box widened by the stencil half-width in x, y and z.
hpsi_status mesh_items_part(hpsi_mesh *m, int zb, int ty, int part, const int4 **items, int *nitems) {
  const int key = (2 * zb + (ty == 8 ? 1 : 0)) * 4 + part;
  auto it = m->items_part.find(key);
  if (it == m->items_part.end()) {
    const CellBox &B = m->box;
    const int HAL = 4;
    const int tyn = ty == 8 ? m->tiles_y8 : m->tiles_y;
    const auto &tz = ty == 8 ? m->tile_z8 : m->tile_z;
    // dirty[tile][z - z0(tile)]: plane z of the tile column reads a ghost cell
    std::vector<std::vector<char>> dirty(tz.size());
    for (size_t t = 0; t < tz.size(); ++t)
      if (tz[t].y >= 0) dirty[t].assign(size_t(tz[t].y - tz[t].x + 1), 0);
    for (int r = m->ghost_first; r < m->ghost_first + m->ghost_count; ++r) {
      const int c = m->cell_of_row_h[r];
      const int x = c % B.NX, y = (c / B.NX) % B.NY, z = c / (B.NX * B.NY);
      // tiles whose widened box [x0 - 4, x0 + 16 + 4) x [y0 - 4, y0 + ty + 4) holds (x, y)
      const int bx0 = std::max(0, (x - HAL - (PASS_TILE + HAL - 1)) / PASS_TILE - 1);
      const int bx1 = std::min(m->tiles_x - 1, (x - HAL + HAL) / PASS_TILE + 1);
      const int by0 = std::max(0, (y - HAL - (ty + HAL - 1)) / ty - 1);
      const int by1 = std::min(tyn - 1, (y - HAL + HAL) / ty + 1);
      for (int by = by0; by <= by1; ++by)
        for (int bx = bx0; bx <= bx1; ++bx) {
          const int x0 = HAL + bx * PASS_TILE, y0 = HAL + by * ty;
          if (x < x0 - HAL || x >= x0 + PASS_TILE + HAL || y < y0 - HAL || y >= y0 + ty + HAL) continue;
          const size_t t = size_t(by) * m->tiles_x + bx;
          if (tz[t].y < 0) continue;
          for (int zz = std::max(tz[t].x, z - HAL); zz <= std::min(tz[t].y, z + HAL); ++zz)
            dirty[t][size_t(zz - tz[t].x)] = 1;
        }
    }
    std::vector<int4> v;
    for (int by = 0; by < tyn; ++by)
      for (int bx = 0; bx < m->tiles_x; ++bx) {
        const size_t t = size_t(by) * m->tiles_x + bx;
        const int2 c = tz[t];
        if (c.y < 0) continue;
        int z = c.x;
        while (z <= c.y) {
          const char d = dirty[t][size_t(z - c.x)];
          int e = z;
          while (e <= c.y && dirty[t][size_t(e - c.x)] == d && e - z < zb) ++e;
          if ((part == 1 && !d) || (part == 2 && d)) v.push_back(make_int4(bx, by, z, e));
          z = e;
        }
      }
    std::stable_sort(v.begin(), v.end(), [zb](const int4 &a, const int4 &b) {
      const int za = a.z / zb, zbb = b.z / zb;
      if (za != zbb) return za < zbb;
      if (a.y != b.y) return a.y < b.y;
      return a.x < b.x;
    });
    int4 *d = nullptr;
    hpsi_status s = dev_alloc(reinterpret_cast<void **>(&d), std::max<size_t>(1, v.size()) * sizeof(int4));
    if (s) return s;
    if (!v.empty()) HPSI_TRY_CUDA(cudaMemcpy(d, v.data(), v.size() * sizeof(int4), cudaMemcpyHostToDevice));
    it = m->items_part.emplace(key, std::make_pair(d, int(v.size()))).first;
  }
  *items = it->second.first;
  *nitems = it->second.second;
  return HPSI_OK;
}

// Per (16 x 8 tile column, cell plane) of the padded box, bit s set when star
// segment s of the tile's halo plane (star cells 8 s .. 8 s + 7 in the order
// of the blocked pass: 4 rows of 16 above, 8 rows of 24, 4 rows of 16 below,
// HAL = 4) maps to eight consecutive rows of the batch through `src`.
static std::vector<unsigned long long> seg_mask_table(const hpsi_mesh *m, const std::vector<int> &src) {
  const CellBox &B = m->box;
  const int HAL = 4, TX = 16, TY = 8, HX = TX + 2 * HAL;
  std::vector<unsigned long long> t(size_t(m->tiles_y8) * m->tiles_x * B.NZ, 0ull);
  for (int by = 0; by < m->tiles_y8; ++by)
    for (int bx = 0; bx < m->tiles_x; ++bx) {
      const int cx0 = HAL + bx * TX, cy0 = HAL + by * TY;
      for (int q = 0; q < B.NZ; ++q) {
        unsigned long long mask = 0;
        for (int sgi = 0; sgi < 40; ++sgi) {
          int first = -1;
          bool ok = true;
          for (int k = 0; k < 8 && ok; ++k) {
            int i = 8 * sgi + k, hx, hy;  // star cell -> halo-plane coordinates
            if (i < HAL * TX) {
              hy = i / TX;
              hx = HAL + i % TX;
            } else if ((i -= HAL * TX) < TY * HX) {
              hy = HAL + i / HX;
              hx = i % HX;
            } else {
              i -= TY * HX;
              hy = HAL + TY + i / TX;
              hx = HAL + i % TX;
            }
            const int x = cx0 - HAL + hx, y = cy0 - HAL + hy;
            const int r = (x < 0 || y < 0 || x >= B.NX || y >= B.NY) ? -1
                                                                      : src[(size_t(q) * B.NY + y) * B.NX + x];
            if (k == 0) first = r;
            ok = r >= 0 && r == first + k;
          }
          if (ok) mask |= 1ull << sgi;
        }
        t[(size_t(by) * m->tiles_x + bx) * B.NZ + q] = mask;
      }
    }
  return t;
}

hpsi_status prepare_tma(hpsi_hamiltonian *h, const int *src_map, long long in_rows, PassShape &shape, PassArgs &a) {
  hpsi_mesh *m = h->mesh;
  a.in_rows = in_rows;
  if (!shape.tma) return HPSI_OK;
  // tables exist for the raw and the zero-boundary maps; periodic images
  // (and their Bloch phases) keep the per-cell copies
  if (a.phase_corr || (src_map != m->d_src_raw && src_map != m->d_src_zero) || m->cell_row_h.empty()) {
    shape.tma = 0;
    return HPSI_OK;
  }
  auto it = m->seg_masks.find(src_map);
  if (it == m->seg_masks.end()) {
    std::vector<int> src(m->cell_row_h);
    if (src_map == m->d_src_zero)
      for (auto &r : src)
        if (r >= m->np) r = -1;
    const std::vector<unsigned long long> t = seg_mask_table(m, src);
    unsigned long long *d = nullptr;
    hpsi_status s = dev_alloc(reinterpret_cast<void **>(&d), std::max<size_t>(1, t.size()) * sizeof(unsigned long long));
    if (s) return s;
    HPSI_TRY_CUDA(cudaMemcpy(d, t.data(), t.size() * sizeof(unsigned long long), cudaMemcpyHostToDevice));
    it = m->seg_masks.emplace(src_map, d).first;
  }
  if (!h->d_err) {
    hpsi_status s = dev_alloc(reinterpret_cast<void **>(&h->d_err), sizeof(int));
    if (s) return s;
    HPSI_TRY_CUDA(cudaMemset(h->d_err, 0, sizeof(int)));
  }
  a.seg_mask = it->second;
  a.seg_tiles_x = m->tiles_x;
  a.err = h->d_err;
  return HPSI_OK;
}

// Build the pass arguments shared by apply and Taylor passes.
void base_pass_args(const hpsi_hamiltonian *h, int terms, const int *src_map, PassArgs &a) {
  const hpsi_mesh *m = h->mesh;
  std::memset(&a, 0, sizeof(a));
  a.box = m->box;
  a.cell_src = src_map;
  a.cell_row = m->d_cell_row;
  a.per_inner = m->d_per_inner;
  a.col_z = m->d_col_z;
  a.np = m->np;
  if ((terms & HPSI_TERM_KINETIC) && h->have_kinetic) {
    std::memcpy(a.wx, h->wx, sizeof(a.wx));
    std::memcpy(a.wy, h->wy, sizeof(a.wy));
    std::memcpy(a.wz, h->wz, sizeof(a.wz));
  }
  for (int k = 0; k < 9; ++k) {
    a.wxf[k] = float(a.wx[k]);
    a.wyf[k] = float(a.wy[k]);
    a.wzf[k] = float(a.wz[k]);
  }
  if (terms & HPSI_TERM_LOCAL_POTENTIAL) {
    a.v_cell = h->d_vcell;
    for (int k = 0; k < 3; ++k) a.fld[k] = h->fld[k];
    a.fld_scale_dev = h->fld_scale_dev;
  }
  a.obs_pol[0] = 0.0;
  a.obs_pol[1] = 0.0;
  a.obs_pol[2] = 1.0;
  if (h->have_pol)
    for (int k = 0; k < 3; ++k) a.obs_pol[k] = h->pol[k];
}

template <typename T>
hpsi_status run_bra(hpsi_hamiltonian *h, const T *psi, long long ld, T *proj, cudaStream_t st) {
  ProjArgs p;
  p.nmat = h->nmat;
  p.max_nproj = h->max_nproj;
  p.mat = h->d_mat;
  p.proj_row = h->d_proj_row;
  p.map = h->d_map;
  p.pt = sizeof(T) == 8 ? static_cast<const void *>(h->d_pt) : static_cast<const void *>(h->d_pt_f);
  p.scal = sizeof(T) == 8 ? static_cast<const void *>(h->d_scal) : static_cast<const void *>(h->d_scal_f);
  p.pt64 = h->d_pt;
  p.scal64 = h->d_scal;
  p.psi = psi;
  p.psi_ld = ld;
  p.proj = proj;
  p.proj_ld = ld;
  p.nprojections = h->nprojections;
  p.min_npoints = h->min_npoints;
  p.phase = h->d_kb_phase ? (sizeof(T) == 8 ? static_cast<const void *>(h->d_kb_phase)
                                            : static_cast<const void *>(h->d_kb_phase_f))
                          : nullptr;
  const int ksplit = bra_ksplit(p, h->mesh->num_sms);
  hpsi_status s = h->bra_partial.ensure(size_t(ksplit) * h->nprojections * ld * 2 * sizeof(double));
  if (s) return s;
  p.partial = static_cast<double *>(h->bra_partial.ptr);
  ProfScope prof(sizeof(T) == 8 ? "bra_fp64" : "bra_fp32", st);
  return launch_bra<T>(p, h->use_tensor_bra, ksplit, st);
}

template <typename T>
hpsi_status run_ket(hpsi_hamiltonian *h, const T *proj, long long ld, int nst, T *out, long long out_ld, int mode,
                    double a_re, double a_im, const T *psi0, long long psi0_ld, double *obs, cudaStream_t st,
                    double *rho_ket = nullptr, const double *rho_w = nullptr, int row_blocks = 0) {
  KetArgs k;
  k.rho_ket = rho_ket;
  k.rho_w = rho_w;
  k.row_blocks = row_blocks;
  k.nk = h->nk;
  k.krows = h->d_krows;
  k.kptr = h->d_kptr;
  k.ent = h->d_kb_ent;
  k.pt = sizeof(T) == 8 ? static_cast<const void *>(h->d_pt) : static_cast<const void *>(h->d_pt_f);
  k.proj = proj;
  k.proj_ld = ld;
  k.out = out;
  k.out_ld = out_ld;
  k.nst = nst;
  k.mode = mode;
  k.a_re = a_re;
  k.a_im = a_im;
  k.psi0 = psi0;
  k.psi0_ld = psi0_ld;
  k.obs = obs;
  k.obs_ld = int(ld);
  k.phase = h->d_kb_phase ? (sizeof(T) == 8 ? static_cast<const void *>(h->d_kb_phase)
                                            : static_cast<const void *>(h->d_kb_phase_f))
                          : nullptr;
  ProfScope prof(sizeof(T) == 8 ? "ket_fp64" : "ket_fp32", st);
  return launch_ket<T>(k, st);
}

// Shape of the fused pass for a batch: the autotuned one when it matches.
PassShape pass_shape(const hpsi_hamiltonian *h, int dtype, long long ld) {
  const auto &t = h->tuned[dtype == HPSI_C128 ? 0 : 1];
  if (t.ld == ld && !std::getenv(dtype == HPSI_C128 ? "HPSI_PASS_SHAPE64" : "HPSI_PASS_SHAPE32")) return t.shape;
  return default_shape(dtype, ld);
}

// Arguments of one fused pass (no launch).  in: rows to stencil; out: result
// rows; psi0: pointwise term of a Horner pass.
template <typename T>
hpsi_status build_pass_args(hpsi_hamiltonian *h, int terms, const int *src_map, const T *in, long long in_ld, T *out,
                            long long out_ld, long long ld, int mode, const T *psi0, long long psi0_ld, double a_re,
                            double a_im, const PassShape &shape, PassArgs &a) {
  base_pass_args(h, terms, src_map, a);
  if (h->mesh->periodic && h->d_src_phase && src_map == h->d_src_phase)
    a.phase_corr = sizeof(T) == 8 ? static_cast<const void *>(h->d_phase) : static_cast<const void *>(h->d_phase_f);
  a.in = in;
  a.in_ld = in_ld;
  a.out = out;
  a.out_ld = out_ld;
  a.mode = mode;
  a.psi0 = psi0;
  a.psi0_ld = psi0_ld;
  a.a_re = a_re;
  a.a_im = a_im;
  a.chunks = int(ld / shape.sc);
  const int ty = shape.blk ? shape.ty : 16;
  a.zb = shape.zb > 0 ? shape.zb : pass_zb(h->mesh, shape, sizeof(T) == 8 ? HPSI_C128 : HPSI_C64, a.chunks);
  return mesh_items(h->mesh, a.zb, ty, &a.items, &a.nitems);
}

// Rows of the tensor the input of a pass holds: the caller's boundary rows
// are read only through the raw map; Taylor workspaces hold np rows.
long long pass_in_rows(const hpsi_hamiltonian *h, const int *src_map) {
  return src_map == h->mesh->d_src_raw ? h->mesh->np_part : h->mesh->np;
}

// Launch a pass with the kernel its shape names.
template <typename T>
hpsi_status launch_pass_any(const PassArgs &a, const PassShape &shape, long long in_rows, cudaStream_t st) {
  (void)in_rows;
  if (shape.blk) return launch_pass_blk<T>(a, shape, st);
  return launch_pass<T>(a, shape, st);
}
template hpsi_status launch_pass_any<double>(const PassArgs &, const PassShape &, long long, cudaStream_t);
template hpsi_status launch_pass_any<float>(const PassArgs &, const PassShape &, long long, cudaStream_t);

// Density of a pass output, fused into the pass (blocked kernel) and the ket.
struct RhoSpec {
  const double *w;    // per state weight, ld entries (zero beyond nst)
  double *part;       // [chunks][np]
  double *ket;        // [ceil(nst / 64)][nk]
  bool fused = false;  // set when the pass took it
};

// One fused pass with its KB bra before and ket after.
template <typename T>
hpsi_status run_pass(hpsi_hamiltonian *h, int terms, const int *src_map, const T *in, long long in_ld, T *out,
                     long long out_ld, long long ld, int mode, const T *psi0, long long psi0_ld, double a_re,
                     double a_im, double *obs_partial, int *ncta_out, cudaStream_t st, RhoSpec *rho = nullptr,
                     int points = 0) {
  PassArgs a;
  const int dtype = sizeof(T) == 8 ? HPSI_C128 : HPSI_C64;
  PassShape shape = pass_shape(h, dtype, ld);
  hpsi_status si = build_pass_args<T>(h, terms, src_map, in, in_ld, out, out_ld, ld, mode, psi0, psi0_ld, a_re,
                                      a_im, shape, a);
  if (si) return si;
  if (shape.blk) {
    PassArgs chk = a;
    if (obs_partial) chk.obs = obs_partial;
    if (obs_partial && !psi0) chk.psi0 = in, chk.psi0_ld = in_ld;
    if (!blk_pass_eligible<T>(chk, ld, shape.sc)) {
      shape = legacy_shape(dtype, ld);
      si = build_pass_args<T>(h, terms, src_map, in, in_ld, out, out_ld, ld, mode, psi0, psi0_ld, a_re, a_im, shape,
                              a);
      if (si) return si;
    }
  }
  if (shape.blk) {
    si = prepare_tma(h, src_map, pass_in_rows(h, src_map), shape, a);
    if (si) return si;
  } else {
    a.in_rows = pass_in_rows(h, src_map);
  }
  if (points != 0) {
    // one part of a domain-parallel mesh (no KB term, no observables)
    const int ty = shape.blk ? shape.ty : 16;
    si = mesh_items_part(h->mesh, a.zb, ty, points, &a.items, &a.nitems);
    if (si) return si;
  }
  const bool nl = (terms & HPSI_TERM_NON_LOCAL_POTENTIAL) && h->nmat > 0;
  // The bra reads only psi, like the pass: it runs on the handle's side
  // stream, forked from and joined back into `st` (a legal fork/join inside a
  // stream capture too), so that its CTAs fill the SMs the pass leaves idle.
  bool forked = false;
  if (nl) {
    const size_t pbytes = size_t(h->nprojections) * ld * 2 * sizeof(T);
    hpsi_status s = h->projbuf.ensure(pbytes);
    if (s) return s;
    if (h->overlap_bra) {
      s = h->ensure_bra_stream();
      if (s) return s;
      forked = true;
    }
  }
  if (obs_partial) {
    a.obs = obs_partial;
    a.obs_ld = int(ld);
  }
  if (ncta_out) *ncta_out = a.nitems;
  if (obs_partial && !psi0) a.psi0 = in, a.psi0_ld = in_ld;
  if (rho && shape.blk && mode == PASS_HORNER && !obs_partial) {
    a.rho_part = rho->part;
    a.rho_w = rho->w;
    rho->fused = true;
  }
  const bool rho_fused = rho && rho->fused;
  // with the bra on its side stream the pass goes first, on the handle's
  // high-priority stream: the block scheduler hands freed SMs to pending pass
  // CTAs before bra CTAs (a pass CTA fills an SM's shared memory, so the two
  // never share an SM), and the bra mostly fills the pass's last, partial wave
  const bool pass_side = forked && h->prio_pass;
  if (forked) HPSI_TRY_CUDA(cudaEventRecord(h->bra_fork, st));
  cudaStream_t pst = st;
  if (pass_side) {
    HPSI_TRY_CUDA(cudaStreamWaitEvent(h->pass_stream, h->bra_fork, 0));
    pst = h->pass_stream;
  }
  hpsi_status sp = HPSI_OK;
  {
    ProfScope prof(sizeof(T) == 8 ? "pass_fp64" : "pass_fp32", pst);
    sp = launch_pass_any<T>(a, shape, pass_in_rows(h, src_map), pst);
  }
  if (pass_side) HPSI_TRY_CUDA(cudaEventRecord(h->pass_join, pst));
  hpsi_status sb = HPSI_OK;
  if (nl) {
    cudaStream_t bst = st;
    if (forked) {
      HPSI_TRY_CUDA(cudaStreamWaitEvent(h->bra_stream, h->bra_fork, 0));
      bst = h->bra_stream;
    }
    // the bra reads only psi, like the pass
    sb = run_bra<T>(h, in, in_ld, static_cast<T *>(h->projbuf.ptr), bst);
    if (forked) HPSI_TRY_CUDA(cudaEventRecord(h->bra_join, bst));
  }
  if (pass_side) HPSI_TRY_CUDA(cudaStreamWaitEvent(st, h->pass_join, 0));
  if (forked) HPSI_TRY_CUDA(cudaStreamWaitEvent(st, h->bra_join, 0));
  if (sp) return sp;
  if (sb) return sb;
  if (nl) {
    double *kobs = nullptr;
    if (obs_partial) {
      hpsi_status s = h->ketobs.ensure(size_t(ket_row_blocks(h->nk)) * ld * 2 * sizeof(double));
      if (s) return s;
      kobs = static_cast<double *>(h->ketobs.ptr);
    }
    hpsi_status s = run_ket<T>(h, static_cast<const T *>(h->projbuf.ptr), ld, int(ld), out, out_ld, mode, a_re, a_im,
                               static_cast<const T *>(a.psi0), a.psi0_ld, kobs, st, rho_fused ? rho->ket : nullptr,
                               rho_fused ? rho->w : nullptr);
    if (s) return s;
  }
  return HPSI_OK;
}

template hpsi_status build_pass_args<double>(hpsi_hamiltonian *, int, const int *, const double *, long long,
                                             double *, long long, long long, int, const double *, long long, double,
                                             double, const PassShape &, PassArgs &);
template hpsi_status build_pass_args<float>(hpsi_hamiltonian *, int, const int *, const float *, long long, float *,
                                            long long, long long, int, const float *, long long, double, double,
                                            const PassShape &, PassArgs &);
template hpsi_status run_bra<double>(hpsi_hamiltonian *, const double *, long long, double *, cudaStream_t);
template hpsi_status run_bra<float>(hpsi_hamiltonian *, const float *, long long, float *, cudaStream_t);
template hpsi_status run_ket<double>(hpsi_hamiltonian *, const double *, long long, int, double *, long long, int,
                                     double, double, const double *, long long, double *, cudaStream_t, double *,
                                     const double *, int);
template hpsi_status run_ket<float>(hpsi_hamiltonian *, const float *, long long, int, float *, long long, int,
                                    double, double, const float *, long long, double *, cudaStream_t, double *,
                                    const double *, int);

const int *load_map(const hpsi_hamiltonian *h, int set_bc) {
  const hpsi_mesh *m = h->mesh;
  if (!set_bc) return m->d_src_raw;
  if (m->periodic) return h->d_src_phase ? h->d_src_phase : m->d_src_per;
  return m->d_src_zero;
}

// size of the observables partial buffer for a pass over ld states
size_t obs_partial_bytes(hpsi_hamiltonian *h, long long ld) {
  size_t n = 0;
  for (int dt : {HPSI_C128, HPSI_C64}) {
    const PassShape sh = pass_shape(h, dt, ld);
    const int4 *items;
    int nitems = 0;
    const int ty = sh.blk ? sh.ty : 16;
    const int zb = sh.zb > 0 ? sh.zb : pass_zb(h->mesh, sh, dt, int(ld / sh.sc));
    if (mesh_items(h->mesh, zb, ty, &items, &nitems) == HPSI_OK)
      n = std::max(n, size_t(nitems));
    const PassShape lg = legacy_shape(dt, ld);
    if (mesh_items(h->mesh, choose_zb(h->mesh, int(ld / lg.sc)), &items, &nitems) == HPSI_OK)
      n = std::max(n, size_t(nitems));
  }
  return std::max<size_t>(n, 1) * ld * 6 * sizeof(double);
}

// Allocate every workspace a Taylor step touches (so that a step can be
// captured in a CUDA graph without allocating).
hpsi_status prepare_taylor_workspaces(hpsi_hamiltonian *h, long long ld, size_t elem, bool obs) {
  hpsi_mesh *m = h->mesh;
  const size_t ubytes = size_t(m->np) * ld * 2 * elem;
  for (auto &w : h->u) {
    hpsi_status s = w.ensure(ubytes);
    if (s) return s;
  }
  if (obs) {
    hpsi_status s = h->obsbuf.ensure(obs_partial_bytes(h, ld));
    if (s) return s;
    s = h->small.ensure(3 * size_t(ld) * sizeof(double));
    if (s) return s;
  }
  if (h->nmat > 0) {
    hpsi_status s = h->projbuf.ensure(size_t(h->nprojections) * ld * 2 * elem);
    if (s) return s;
    ProjArgs p;
    std::memset(&p, 0, sizeof(p));
    p.nmat = h->nmat;
    p.psi_ld = ld;
    p.min_npoints = h->min_npoints;
    s = h->bra_partial.ensure(size_t(bra_ksplit(p, m->num_sms)) * h->nprojections * ld * 2 * sizeof(double));
    if (s) return s;
    if (obs) {
      s = h->ketobs.ensure(size_t(ket_row_blocks(h->nk)) * ld * 2 * sizeof(double));
      if (s) return s;
    }
  }
  return HPSI_OK;
}

template <typename T>
hpsi_status apply_h_dev(hpsi_hamiltonian *h, const T *psi, long long ld, T *hpsi, long long ldo, int terms,
                        int set_bc, cudaStream_t st) {
  return run_pass<T>(h, terms, load_map(h, set_bc), psi, ld, hpsi, ldo, ld, PASS_APPLY, nullptr, 0, 0.0, 0.0,
                     nullptr, nullptr, st);
}

// Horner form of the order-K Taylor polynomial, K fused passes; with `rho`
// the last pass (and its ket) also writes the density partials of the result.
template <typename T>
hpsi_status taylor_dev_impl(hpsi_hamiltonian *h, T *psi, long long ld, int nst, double dt_re, double dt_im,
                            int order, double *obs_dev, cudaStream_t st, RhoSpec *rho) {
  hpsi_mesh *m = h->mesh;
  const size_t ubytes = size_t(m->np) * ld * 2 * sizeof(T);
  for (auto &w : h->u) {
    hpsi_status s = w.ensure(ubytes);
    if (s) return s;
  }
  double *obs_partial = nullptr;
  if (obs_dev) {
    hpsi_status s = h->obsbuf.ensure(obs_partial_bytes(h, ld));
    if (s) return s;
    obs_partial = static_cast<double *>(h->obsbuf.ptr);
  }
  const int *map = load_map(h, 1);
  T *u0 = static_cast<T *>(h->u[0].ptr), *u1 = static_cast<T *>(h->u[1].ptr);
  const T *in = psi;
  long long in_ld = ld;
  int ncta = 0;
  for (int k = order; k >= 1; --k) {
    // a_k = -i dt / k
    const double are = dt_im / k, aim = -dt_re / k;
    T *out = (k == 1 && order > 1) ? psi : ((order - k) % 2 == 0 ? u0 : u1);
    const long long out_ld = (out == psi) ? ld : ld;
    hpsi_status s = run_pass<T>(h, HPSI_TERM_ALL, map, in, in_ld, out, out_ld, ld, PASS_HORNER, psi, ld, are, aim,
                                k == order ? obs_partial : nullptr, k == order ? &ncta : nullptr, st,
                                k == 1 ? rho : nullptr);
    if (s) return s;
    in = out;
    in_ld = out_ld;
  }
  if (order == 1) {
    const long long n = (long long)m->np * nst;
    copy_rows_kernel<T><<<unsigned((n + 255) / 256), 256, 0, st>>>(u0, ld, psi, ld, m->np, nst);
    HPSI_CHECK_LAUNCH();
  }
  if (obs_dev) {
    const bool nl = h->nmat > 0 && h->nk > 0;
    hpsi_status s = launch_obs_finalize(obs_partial, ncta, int(ld), nst, m->box.h[0] * m->box.h[1] * m->box.h[2],
                                        nl ? static_cast<const double *>(h->ketobs.ptr) : nullptr,
                                        nl ? ket_row_blocks(h->nk) : 0, obs_dev, st);
    if (s) return s;
  }
  return HPSI_OK;
}

template <typename T>
hpsi_status taylor_dev(hpsi_hamiltonian *h, T *psi, long long ld, int nst, double dt_re, double dt_im, int order,
                       double *obs_dev, cudaStream_t st) {
  return taylor_dev_impl<T>(h, psi, ld, nst, dt_re, dt_im, order, obs_dev, st, nullptr);
}

template hpsi_status apply_h_dev<double>(hpsi_hamiltonian *, const double *, long long, double *, long long, int, int,
                                         cudaStream_t);
template hpsi_status apply_h_dev<float>(hpsi_hamiltonian *, const float *, long long, float *, long long, int, int,
                                        cudaStream_t);
template hpsi_status taylor_dev<double>(hpsi_hamiltonian *, double *, long long, int, double, double, int, double *,
                                        cudaStream_t);
template hpsi_status taylor_dev<float>(hpsi_hamiltonian *, float *, long long, int, double, double, int, double *,
                                       cudaStream_t);

// Host-pointer staging: copy a host batch into a device workspace.
hpsi_status stage_batch(Workspace &ws, const hpsi_batch *b, int rows, bool copy_in, cudaStream_t st, void **dev) {
  const size_t esz = b->dtype == HPSI_C128 ? 16 : 8;
  const size_t bytes = size_t(rows) * b->ld * esz;
  hpsi_status s = ws.ensure(bytes);
  if (s) return s;
  if (copy_in) HPSI_TRY_CUDA(cudaMemcpyAsync(ws.ptr, b->ptr, bytes, cudaMemcpyHostToDevice, st));
  *dev = ws.ptr;
  return HPSI_OK;
}

// H psi for host batches, pipelined over state slabs: the copy-in of slab
// i + 1, the passes of slab i and the copy-out of slab i - 1 run at once on
// three streams (two copy engines and the SMs), double-buffered on the
// device.  Rows copied in: np when the boundary condition is applied (the
// boundary rows are then never read), np_part otherwise.
template <typename T>
hpsi_status apply_h_host_pipelined(hpsi_hamiltonian *h, const hpsi_batch *psi, hpsi_batch *hpsi, int terms,
                                   int set_bc, const std::vector<long long> &widths, cudaStream_t st) {
  hpsi_mesh *m = h->mesh;
  const size_t esz = 2 * sizeof(T);
  const long long ld = psi->ld, ldo = hpsi->ld;
  const int nslab = int(widths.size());
  const long long wmax = *std::max_element(widths.begin(), widths.end());
  const int rows_in = set_bc ? m->np : m->np_part;
  const size_t in_bytes = size_t(m->np_part) * wmax * esz, out_bytes = size_t(m->np) * wmax * esz;
  hpsi_status s = h->slab_in.ensure(2 * in_bytes);
  if (!s) s = h->slab_out.ensure(2 * out_bytes);
  if (s) return s;
  if (!h->xfer_in) {
    HPSI_TRY_CUDA(cudaStreamCreateWithFlags(&h->xfer_in, cudaStreamNonBlocking));
    HPSI_TRY_CUDA(cudaStreamCreateWithFlags(&h->xfer_out, cudaStreamNonBlocking));
    for (auto &e : h->xev) HPSI_TRY_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  cudaEvent_t *in_done = h->xev, *comp_done = h->xev + 2, *out_done = h->xev + 4;
  // the copy streams start after the work already queued on st
  HPSI_TRY_CUDA(cudaEventRecord(comp_done[0], st));
  HPSI_TRY_CUDA(cudaStreamWaitEvent(h->xfer_in, comp_done[0], 0));
  HPSI_TRY_CUDA(cudaStreamWaitEvent(h->xfer_out, comp_done[0], 0));
  long long c0 = 0;  // first state of slab i
  for (int i = 0; i < nslab; ++i) {
    const int b = i & 1;
    const long long w = widths[i];
    T *din = reinterpret_cast<T *>(static_cast<char *>(h->slab_in.ptr) + b * in_bytes);
    T *dout = reinterpret_cast<T *>(static_cast<char *>(h->slab_out.ptr) + b * out_bytes);
    const size_t col = size_t(c0) * esz;
    c0 += w;
    if (i >= 2) HPSI_TRY_CUDA(cudaStreamWaitEvent(h->xfer_in, comp_done[b], 0));
    HPSI_TRY_CUDA(cudaMemcpy2DAsync(din, w * esz, static_cast<const char *>(psi->ptr) + col, ld * esz, w * esz,
                                    rows_in, cudaMemcpyHostToDevice, h->xfer_in));
    HPSI_TRY_CUDA(cudaEventRecord(in_done[b], h->xfer_in));
    HPSI_TRY_CUDA(cudaStreamWaitEvent(st, in_done[b], 0));
    if (i >= 2) HPSI_TRY_CUDA(cudaStreamWaitEvent(st, out_done[b], 0));
    s = apply_h_dev<T>(h, din, w, dout, w, terms, set_bc, st);
    if (s) return s;
    HPSI_TRY_CUDA(cudaEventRecord(comp_done[b], st));
    HPSI_TRY_CUDA(cudaStreamWaitEvent(h->xfer_out, comp_done[b], 0));
    HPSI_TRY_CUDA(cudaMemcpy2DAsync(static_cast<char *>(hpsi->ptr) + col, ldo * esz, dout, w * esz, w * esz, m->np,
                                    cudaMemcpyDeviceToHost, h->xfer_out));
    HPSI_TRY_CUDA(cudaEventRecord(out_done[b], h->xfer_out));
  }
  HPSI_TRY_CUDA(cudaStreamSynchronize(h->xfer_out));
  HPSI_TRY_CUDA(cudaStreamSynchronize(st));
  return HPSI_OK;
}

// State slabs of the host pipeline (widths in states, each a multiple of the
// blocked pass's chunk, summing to the batch width); empty when the batch does
// not split.  Default: the most equal slabs, at most 4.  Measured on
// 904,089 x 128 complex128 (two 1.85 GB copies at 53-56 GB/s each way): 2
// slabs 55.0 ms, 4 slabs 46.7 ms, 8 slabs 53.5 ms (the strided copies of
// narrow slabs lose bandwidth).  Tapered splits, which shorten the exposed
// first copy-in and last copy-out, measured slower still: 16,32,32,32,16
// 47.2 ms, 8,24,32,32,24,8 49.2 ms, 24,40,40,24 51.3 ms, 16,48,48,16 50.6 ms
// against 46.4 ms for 4 x 32 (copies of 512-byte row pieces run fastest).
// HPSI_HOST_SLAB_WIDTHS (a comma-separated list of widths) overrides the split
// when it is valid for the batch.
std::vector<long long> pipeline_slabs(const hpsi_batch *psi, const hpsi_batch *hpsi) {
  const long long chunk = psi->dtype == HPSI_C128 ? blk_chunk_states<double>() : blk_chunk_states<float>();
  std::vector<long long> out;
  if (psi->ld != hpsi->ld || psi->nst != psi->ld) return out;
  if (const char *e = std::getenv("HPSI_HOST_SLAB_WIDTHS")) {
    long long sum = 0;
    bool ok = true;
    for (const char *q = e; *q;) {
      char *end = nullptr;
      const long long w = std::strtoll(q, &end, 10);
      if (end == q || w <= 0 || w % chunk != 0) {
        ok = false;
        break;
      }
      out.push_back(w);
      sum += w;
      q = *end == ',' ? end + 1 : end;
    }
    if (ok && sum == psi->ld && out.size() >= 2) return out;
    out.clear();
  }
  int maxslab = 4;
  if (const char *e = std::getenv("HPSI_HOST_SLABS")) maxslab = std::max(1, std::atoi(e));
  for (int nslab = maxslab; nslab >= 2; --nslab)
    if (psi->ld % (nslab * chunk) == 0) return std::vector<long long>(nslab, psi->ld / nslab);
  return out;
}

}  // namespace hpsi

extern "C" {

hpsi_status hpsi_apply_h(hpsi_hamiltonian *h, const hpsi_batch *psi, hpsi_batch *hpsi, int32_t terms,
                         int32_t set_bc, void *stream) {
  if (!h) return HPSI_ERR_ARG;
  hpsi_mesh *m = h->mesh;
  hpsi_status s = check_batch(m, psi, m->np_part, "hpsi_apply_h(psi)");
  if (!s) s = check_batch(m, hpsi, m->np, "hpsi_apply_h(hpsi)");
  if (s) return s;
  if (psi->dtype != hpsi->dtype || psi->nst != hpsi->nst) {
    set_error("hpsi_apply_h: psi and hpsi differ in dtype or nst");
    return HPSI_ERR_ARG;
  }
  if ((terms & HPSI_TERM_KINETIC) && !h->have_kinetic) {
    set_error("hpsi_apply_h: kinetic weights not set");
    return HPSI_ERR_STATE;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const bool din = is_device_ptr(psi->ptr), dout = is_device_ptr(hpsi->ptr);
  if (!din && !dout) {
    const std::vector<long long> widths = pipeline_slabs(psi, hpsi);
    if (!widths.empty())
      return psi->dtype == HPSI_C128 ? apply_h_host_pipelined<double>(h, psi, hpsi, terms, set_bc, widths, st)
                                     : apply_h_host_pipelined<float>(h, psi, hpsi, terms, set_bc, widths, st);
  }
  const void *pin = psi->ptr;
  void *pout = hpsi->ptr;
  long long ldi = psi->ld, ldo = hpsi->ld;
  if (!din) {
    void *d;
    s = stage_batch(m->stage_in, psi, m->np_part, true, st, &d);
    if (s) return s;
    pin = d;
  }
  if (!dout) {
    void *d;
    s = stage_batch(m->stage_out, hpsi, m->np, false, st, &d);
    if (s) return s;
    pout = d;
  }
  if (psi->dtype == HPSI_C128)
    s = apply_h_dev<double>(h, static_cast<const double *>(pin), ldi, static_cast<double *>(pout), ldo, terms, set_bc,
                            st);
  else
    s = apply_h_dev<float>(h, static_cast<const float *>(pin), ldi, static_cast<float *>(pout), ldo, terms, set_bc,
                           st);
  if (s) return s;
  if (!dout) {
    const size_t esz = hpsi->dtype == HPSI_C128 ? 16 : 8;
    HPSI_TRY_CUDA(cudaMemcpyAsync(hpsi->ptr, pout, size_t(m->np) * ldo * esz, cudaMemcpyDeviceToHost, st));
  }
  if (!din || !dout) HPSI_TRY_CUDA(cudaStreamSynchronize(st));
  return HPSI_OK;
}

hpsi_status hpsi_boundaries_set(hpsi_hamiltonian *h, hpsi_batch *psi, void *stream) {
  if (!h) return HPSI_ERR_ARG;
  hpsi_mesh *m = h->mesh;
  hpsi_status s = check_batch(m, psi, m->np_part, "hpsi_boundaries_set");
  if (s) return s;
  if (!is_device_ptr(psi->ptr)) {
    set_error("hpsi_boundaries_set: device batch expected");
    return HPSI_ERR_ARG;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int nb = m->np_part - m->np;
  if (nb == 0) return HPSI_OK;
  const long long n = (long long)nb * psi->ld;
  if (psi->dtype == HPSI_C128)
    boundaries_kernel<double><<<unsigned((n + 255) / 256), 256, 0, st>>>(
        static_cast<double *>(psi->ptr), psi->ld, m->np, nb, m->d_per_inner, h->d_phase, m->periodic);
  else
    boundaries_kernel<float><<<unsigned((n + 255) / 256), 256, 0, st>>>(
        static_cast<float *>(psi->ptr), psi->ld, m->np, nb, m->d_per_inner, h->d_phase_f, m->periodic);
  HPSI_CHECK_LAUNCH();
  return HPSI_OK;
}

hpsi_status hpsi_taylor_step(hpsi_hamiltonian *h, hpsi_batch *psi, double dt_re, double dt_im, int32_t order,
                             double *energy, double *dipole, double *norm2, void *stream) {
  if (!h) return HPSI_ERR_ARG;
  hpsi_mesh *m = h->mesh;
  hpsi_status s = check_batch(m, psi, m->np, "hpsi_taylor_step");
  if (s) return s;
  if (order < 1 || order > 32) {
    set_error("hpsi_taylor_step: order must be 1..32");
    return HPSI_ERR_ARG;
  }
  if (!h->have_kinetic) {
    set_error("hpsi_taylor_step: kinetic weights not set");
    return HPSI_ERR_STATE;
  }
  if (!std::isfinite(dt_re) || !std::isfinite(dt_im)) return HPSI_ERR_ARG;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const bool want_obs = energy || dipole || norm2;
  double *obs_dev = nullptr;
  if (want_obs) {
    s = h->small.ensure(3 * size_t(psi->nst) * sizeof(double));
    if (s) return s;
    obs_dev = static_cast<double *>(h->small.ptr);
  }
  const bool dev = is_device_ptr(psi->ptr);
  void *p = psi->ptr;
  if (!dev) {
    s = stage_batch(m->stage_in, psi, m->np, true, st, &p);
    if (s) return s;
  }
  if (psi->dtype == HPSI_C128)
    s = taylor_dev<double>(h, static_cast<double *>(p), psi->ld, psi->nst, dt_re, dt_im, order, obs_dev, st);
  else
    s = taylor_dev<float>(h, static_cast<float *>(p), psi->ld, psi->nst, dt_re, dt_im, order, obs_dev, st);
  if (s) return s;
  if (!dev) {
    const size_t esz = psi->dtype == HPSI_C128 ? 16 : 8;
    HPSI_TRY_CUDA(cudaMemcpyAsync(psi->ptr, p, size_t(m->np) * psi->ld * esz, cudaMemcpyDeviceToHost, st));
  }
  if (want_obs) {
    std::vector<double> hv(3 * size_t(psi->nst));
    HPSI_TRY_CUDA(cudaMemcpyAsync(hv.data(), obs_dev, hv.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    HPSI_TRY_CUDA(cudaStreamSynchronize(st));
    bool finite = true;
    for (double x : hv) finite = finite && std::isfinite(x);
    const int n = psi->nst;
    if (energy) std::memcpy(energy, hv.data(), n * sizeof(double));
    if (norm2) std::memcpy(norm2, hv.data() + n, n * sizeof(double));
    if (dipole) std::memcpy(dipole, hv.data() + 2 * n, n * sizeof(double));
    if (!finite) {
      set_error("hpsi_taylor_step: non-finite observable (NaN/Inf in the batch)");
      return HPSI_ERR_NONFINITE;
    }
  } else if (!dev) {
    HPSI_TRY_CUDA(cudaStreamSynchronize(st));
  }
  return HPSI_OK;
}

hpsi_status hpsi_taylor_step_density(hpsi_hamiltonian *h, hpsi_batch *psi, double dt_re, double dt_im, int32_t order,
                                     const double *weight, double *rho, int32_t accumulate, void *stream) {
  if (!h || !weight || !rho) return HPSI_ERR_ARG;
  hpsi_mesh *m = h->mesh;
  hpsi_status s = check_batch(m, psi, m->np, "hpsi_taylor_step_density");
  if (s) return s;
  if (order < 1 || order > 32 || !std::isfinite(dt_re) || !std::isfinite(dt_im)) {
    set_error("hpsi_taylor_step_density: order must be 1..32 and dt finite");
    return HPSI_ERR_ARG;
  }
  if (!h->have_kinetic) {
    set_error("hpsi_taylor_step_density: kinetic weights not set");
    return HPSI_ERR_STATE;
  }
  if (!is_device_ptr(psi->ptr) || !is_device_ptr(rho)) {
    set_error("hpsi_taylor_step_density: device batch and density expected");
    return HPSI_ERR_ARG;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const long long ld = psi->ld;
  const PassShape sh = pass_shape(h, psi->dtype, ld);
  const int chunks = int(ld / std::max(1, sh.sc)) + 1;
  const int kxb = (psi->nst + 63) / 64;
  const size_t nw = size_t(ld), npart = size_t(chunks) * m->np, nket = size_t(kxb) * std::max(1, h->nk);
  s = h->rhobuf.ensure((nw + npart + nket) * sizeof(double));
  if (s) return s;
  double *w = static_cast<double *>(h->rhobuf.ptr);
  std::vector<double> wh(nw, 0.0);
  for (int i = 0; i < psi->nst; ++i) {
    if (!std::isfinite(weight[i])) {
      set_error("hpsi_taylor_step_density: non-finite weight");
      return HPSI_ERR_NONFINITE;
    }
    wh[i] = weight[i];
  }
  HPSI_TRY_CUDA(cudaMemcpyAsync(w, wh.data(), nw * sizeof(double), cudaMemcpyHostToDevice, st));
  RhoSpec R;
  R.w = w;
  R.part = w + nw;
  R.ket = R.part + npart;
  // The fused form (density partials written by the last Horner pass, the
  // ket's rows from their final values) measured slower on the 904,089-point
  // sphere with 128 states than the step followed by the density pass
  // (FP64 +0.42 ms against +0.29 ms per step, FP32 +0.27 against +0.17): its
  // cross-lane sums share the MIO pipe with the stencil's shared-memory
  // loads.  The default is therefore the separate pass; fuse_density selects
  // the fused form.
  RhoSpec *rp = h->fuse_density ? &R : nullptr;
  if (psi->dtype == HPSI_C128)
    s = taylor_dev_impl<double>(h, static_cast<double *>(psi->ptr), ld, psi->nst, dt_re, dt_im, order, nullptr, st,
                                rp);
  else
    s = taylor_dev_impl<float>(h, static_cast<float *>(psi->ptr), ld, psi->nst, dt_re, dt_im, order, nullptr, st,
                               rp);
  if (s) return s;
  if (R.fused) {
    const bool kb = h->nmat > 0 && h->nk > 0;
    rho_finalize_kernel<<<(m->np + 255) / 256, 256, 0, st>>>(R.part, int(ld / sh.sc), R.ket, kxb, h->nk,
                                                             kb ? h->d_kidx : nullptr, m->np, accumulate ? 1 : 0,
                                                             rho);
    g_launches++;
    HPSI_CHECK_LAUNCH();
  } else {
    // the density kernel reads the propagated batch once more (the default,
    // and widths the register-blocked pass does not take)
    if (psi->dtype == HPSI_C128)
      s = launch_density<double>(static_cast<const double *>(psi->ptr), ld, m->np, psi->nst, w, rho,
                                 accumulate != 0, st);
    else
      s = launch_density<float>(static_cast<const float *>(psi->ptr), ld, m->np, psi->nst, w, rho,
                                accumulate != 0, st);
    if (s) return s;
  }
  return HPSI_OK;
}

// ---------------------------------------------------------------------------
hpsi_status hpsi_density_accumulate(hpsi_mesh *m, const hpsi_batch *psi, const double *weight, double *rho,
                                    int32_t accumulate, void *stream) {
  if (!m || !weight || !rho) return HPSI_ERR_ARG;
  hpsi_status s = check_batch(m, psi, m->np, "hpsi_density_accumulate");
  if (s) return s;
  if (!is_device_ptr(psi->ptr) || !is_device_ptr(rho)) {
    set_error("hpsi_density_accumulate: device batch and density expected");
    return HPSI_ERR_ARG;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  s = m->scratch2.ensure(size_t(psi->nst) * sizeof(double));
  if (s) return s;
  double *w = static_cast<double *>(m->scratch2.ptr);
  HPSI_TRY_CUDA(cudaMemcpyAsync(w, weight, size_t(psi->nst) * sizeof(double), cudaMemcpyHostToDevice, st));
  if (psi->dtype == HPSI_C128)
    return launch_density<double>(static_cast<const double *>(psi->ptr), psi->ld, m->np, psi->nst, w, rho,
                                  accumulate != 0, st);
  return launch_density<float>(static_cast<const float *>(psi->ptr), psi->ld, m->np, psi->nst, w, rho,
                               accumulate != 0, st);
}

hpsi_status hpsi_nrm2(hpsi_mesh *m, const hpsi_batch *psi, double *out, void *stream) {
  if (!m || !out) return HPSI_ERR_ARG;
  hpsi_status s = check_batch(m, psi, m->np, "hpsi_nrm2");
  if (s) return s;
  if (!is_device_ptr(psi->ptr)) {
    set_error("hpsi_nrm2: device batch expected");
    return HPSI_ERR_ARG;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int nblk = reduce_blocks(m->np);
  const size_t pbytes = size_t(nblk) * psi->nst * 4 * sizeof(double);
  s = m->scratch.ensure(pbytes + 2 * size_t(psi->nst) * sizeof(double));
  if (s) return s;
  double *partial = static_cast<double *>(m->scratch.ptr);
  double *res = partial + size_t(nblk) * psi->nst * 4;
  const double dv = m->box.h[0] * m->box.h[1] * m->box.h[2];
  if (psi->dtype == HPSI_C128)
    s = launch_state_sum<double>(0, static_cast<const double *>(psi->ptr), psi->ld, nullptr, 0, m->np, psi->nst,
                                 partial, nblk, dv, 1, res, st);
  else
    s = launch_state_sum<float>(0, static_cast<const float *>(psi->ptr), psi->ld, nullptr, 0, m->np, psi->nst,
                                partial, nblk, dv, 1, res, st);
  if (s) return s;
  std::vector<double> hv(2 * size_t(psi->nst));
  HPSI_TRY_CUDA(cudaMemcpyAsync(hv.data(), res, hv.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
  HPSI_TRY_CUDA(cudaStreamSynchronize(st));
  for (int i = 0; i < psi->nst; ++i) out[i] = hv[2 * i];
  return HPSI_OK;
}

hpsi_status hpsi_dotp_matrix(hpsi_mesh *m, const hpsi_batch *a, const hpsi_batch *b, double *out, void *stream) {
  if (!m || !out) return HPSI_ERR_ARG;
  hpsi_status s = check_batch(m, a, m->np, "hpsi_dotp_matrix(a)");
  if (!s) s = check_batch(m, b, m->np, "hpsi_dotp_matrix(b)");
  if (s) return s;
  if (a->dtype != b->dtype || a->nst != b->nst) {
    set_error("hpsi_dotp_matrix: a and b differ in dtype or nst");
    return HPSI_ERR_ARG;
  }
  if (!is_device_ptr(a->ptr) || !is_device_ptr(b->ptr)) {
    set_error("hpsi_dotp_matrix: device batches expected");
    return HPSI_ERR_ARG;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int nst = a->nst, splits = gram_splits(m->np);
  const size_t pbytes = size_t(splits) * 4 * nst * nst * sizeof(double);
  s = m->scratch.ensure(pbytes + 2 * size_t(nst) * nst * sizeof(double));
  if (s) return s;
  double *partial = static_cast<double *>(m->scratch.ptr);
  double *S = partial + size_t(splits) * 4 * nst * nst;
  const double dv = m->box.h[0] * m->box.h[1] * m->box.h[2];
  if (a->dtype == HPSI_C128)
    s = launch_gram<double>(static_cast<const double *>(a->ptr), a->ld, static_cast<const double *>(b->ptr), b->ld,
                            m->np, nst, partial, splits, dv, S, st);
  else
    s = launch_gram<float>(static_cast<const float *>(a->ptr), a->ld, static_cast<const float *>(b->ptr), b->ld,
                           m->np, nst, partial, splits, dv, S, st);
  if (s) return s;
  HPSI_TRY_CUDA(cudaMemcpyAsync(out, S, 2 * size_t(nst) * nst * sizeof(double), cudaMemcpyDeviceToHost, st));
  HPSI_TRY_CUDA(cudaStreamSynchronize(st));
  return HPSI_OK;
}

hpsi_status hpsi_orthonormalize_cholesky(hpsi_mesh *m, hpsi_batch *psi, void *stream) {
  if (!m) return HPSI_ERR_ARG;
  hpsi_status s = check_batch(m, psi, m->np, "hpsi_orthonormalize_cholesky");
  if (s) return s;
  if (!is_device_ptr(psi->ptr)) {
    set_error("hpsi_orthonormalize_cholesky: device batch expected");
    return HPSI_ERR_ARG;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int nst = psi->nst, splits = gram_splits(m->np);
  const size_t pbytes = size_t(splits) * 4 * nst * nst * sizeof(double);
  const size_t mbytes = 2 * size_t(nst) * nst * sizeof(double);
  s = m->scratch.ensure(pbytes + 3 * mbytes + 16);
  if (s) return s;
  double *partial = static_cast<double *>(m->scratch.ptr);
  double *S = partial + size_t(splits) * 4 * nst * nst;
  double *U = S + 2 * size_t(nst) * nst;
  double *Uinv = U + 2 * size_t(nst) * nst;
  int *err = reinterpret_cast<int *>(Uinv + 2 * size_t(nst) * nst);
  HPSI_TRY_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));
  const double dv = m->box.h[0] * m->box.h[1] * m->box.h[2];
  if (psi->dtype == HPSI_C128)
    s = launch_gram<double>(static_cast<const double *>(psi->ptr), psi->ld, static_cast<const double *>(psi->ptr),
                            psi->ld, m->np, nst, partial, splits, dv, S, st);
  else
    s = launch_gram<float>(static_cast<const float *>(psi->ptr), psi->ld, static_cast<const float *>(psi->ptr),
                           psi->ld, m->np, nst, partial, splits, dv, S, st);
  if (s) return s;
  s = launch_cholesky_inverse(S, nst, U, Uinv, err, st);
  if (s) return s;
  int herr = 0;
  HPSI_TRY_CUDA(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st));
  HPSI_TRY_CUDA(cudaStreamSynchronize(st));
  if (herr) {
    set_error("hpsi_orthonormalize_cholesky: overlap matrix is not positive definite");
    return HPSI_ERR_ARG;
  }
  if (psi->dtype == HPSI_C128)
    s = launch_trsm_apply<double>(static_cast<double *>(psi->ptr), psi->ld, m->np, nst, Uinv, st);
  else
    s = launch_trsm_apply<float>(static_cast<float *>(psi->ptr), psi->ld, m->np, nst, Uinv, st);
  return s;
}

hpsi_status hpsi_projector_count(const hpsi_hamiltonian *h, int32_t *nprojections) {
  if (!h || !nprojections) return HPSI_ERR_ARG;
  *nprojections = h->nmat > 0 ? h->nprojections : 0;
  return HPSI_OK;
}

// proj must be device memory on a 16-byte boundary (the bra and ket read and
// write whole complex numbers of each row)
static hpsi_status check_proj(const void *proj, const char *what) {
  if (!proj || !is_device_ptr(proj) || reinterpret_cast<uintptr_t>(proj) % 16 != 0) {
    set_error(std::string(what) + ": proj must be device memory on a 16-byte boundary");
    return HPSI_ERR_ARG;
  }
  return HPSI_OK;
}

hpsi_status hpsi_projector_bra(hpsi_hamiltonian *h, const hpsi_batch *psi, void *proj, void *stream) {
  if (!h) return HPSI_ERR_ARG;
  hpsi_status s = check_batch(h->mesh, psi, h->mesh->np, "hpsi_projector_bra(psi)");
  if (s) return s;
  if (h->nmat == 0) return HPSI_OK;
  if (!is_device_ptr(psi->ptr)) {
    set_error("hpsi_projector_bra: psi must be device memory");
    return HPSI_ERR_ARG;
  }
  s = check_proj(proj, "hpsi_projector_bra");
  if (s) return s;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (psi->dtype == HPSI_C128)
    return run_bra<double>(h, static_cast<const double *>(psi->ptr), psi->ld, static_cast<double *>(proj), st);
  return run_bra<float>(h, static_cast<const float *>(psi->ptr), psi->ld, static_cast<float *>(proj), st);
}

hpsi_status hpsi_projector_ket(hpsi_hamiltonian *h, const void *proj, double a_re, double a_im, hpsi_batch *hpsi,
                               void *stream) {
  if (!h) return HPSI_ERR_ARG;
  hpsi_status s = check_batch(h->mesh, hpsi, h->mesh->np, "hpsi_projector_ket(hpsi)");
  if (s) return s;
  if (h->nmat == 0) return HPSI_OK;
  if (!is_device_ptr(hpsi->ptr)) {
    set_error("hpsi_projector_ket: hpsi must be device memory");
    return HPSI_ERR_ARG;
  }
  s = check_proj(proj, "hpsi_projector_ket");
  if (s) return s;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int mode = (a_re == 1.0 && a_im == 0.0) ? PASS_APPLY : PASS_HORNER;
  if (hpsi->dtype == HPSI_C128)
    return run_ket<double>(h, static_cast<const double *>(proj), hpsi->ld, hpsi->nst,
                           static_cast<double *>(hpsi->ptr), hpsi->ld, mode, a_re, a_im, nullptr, 0, nullptr, st);
  return run_ket<float>(h, static_cast<const float *>(proj), hpsi->ld, hpsi->nst, static_cast<float *>(hpsi->ptr),
                        hpsi->ld, mode, a_re, a_im, nullptr, 0, nullptr, st);
}

hpsi_status hpsi_apply_h_horner(hpsi_hamiltonian *h, const hpsi_batch *psi, const hpsi_batch *psi0,
                                hpsi_batch *out, double a_re, double a_im, int32_t terms, int32_t set_bc,
                                void *stream) {
  if (!h) return HPSI_ERR_ARG;
  hpsi_mesh *m = h->mesh;
  hpsi_status s = check_batch(m, psi, m->np_part, "hpsi_apply_h_horner(psi)");
  if (!s) s = check_batch(m, psi0, m->np, "hpsi_apply_h_horner(psi0)");
  if (!s) s = check_batch(m, out, m->np, "hpsi_apply_h_horner(out)");
  if (s) return s;
  if (psi->dtype != out->dtype || psi0->dtype != out->dtype || psi->ld != out->ld || psi0->ld != out->ld ||
      psi->nst != out->nst || psi0->nst != out->nst) {
    set_error("hpsi_apply_h_horner: psi, psi0 and out differ in dtype, ld or nst");
    return HPSI_ERR_ARG;
  }
  if (!is_device_ptr(psi->ptr) || !is_device_ptr(psi0->ptr) || !is_device_ptr(out->ptr)) {
    set_error("hpsi_apply_h_horner: batches must be device memory");
    return HPSI_ERR_ARG;
  }
  if (psi->ptr == out->ptr) {
    set_error("hpsi_apply_h_horner: out must not be psi (the stencil reads neighbours of each row)");
    return HPSI_ERR_ARG;
  }
  if ((terms & HPSI_TERM_KINETIC) && !h->have_kinetic) {
    set_error("hpsi_apply_h_horner: kinetic weights not set");
    return HPSI_ERR_STATE;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const long long ld = out->ld;
  if (out->dtype == HPSI_C128)
    return run_pass<double>(h, terms, load_map(h, set_bc), static_cast<const double *>(psi->ptr), ld,
                            static_cast<double *>(out->ptr), ld, ld, PASS_HORNER,
                            static_cast<const double *>(psi0->ptr), ld, a_re, a_im, nullptr, nullptr, st);
  return run_pass<float>(h, terms, load_map(h, set_bc), static_cast<const float *>(psi->ptr), ld,
                         static_cast<float *>(out->ptr), ld, ld, PASS_HORNER, static_cast<const float *>(psi0->ptr),
                         ld, a_re, a_im, nullptr, nullptr, st);
}


hpsi_status hpsi_mesh_set_ghost_rows(hpsi_mesh *m, int32_t first, int32_t count) {
  if (!m || count < 0 || (count > 0 && (first < m->np || first + (long long)count > m->np_part))) {
    set_error("hpsi_mesh_set_ghost_rows: the ghost rows must lie in [np, np_part)");
    return HPSI_ERR_ARG;
  }
  for (auto &kv : m->items_part) dev_free(kv.second.first);
  m->items_part.clear();
  m->ghost_first = count ? first : 0;
  m->ghost_count = count;
  return HPSI_OK;
}

static hpsi_status check_points(const hpsi_hamiltonian *h, int32_t terms, int32_t points, const char *who) {
  if (points < 0 || points > 2) {
    set_error(std::string(who) + ": points must be HPSI_POINTS_ALL, _INNER or _OUTER");
    return HPSI_ERR_ARG;
  }
  if (points != 0 && (terms & HPSI_TERM_NON_LOCAL_POTENTIAL) && h->nmat > 0) {
    set_error(std::string(who) +
              ": the KB term is added once after both parts (hpsi_projector_bra / hpsi_projector_ket)");
    return HPSI_ERR_ARG;
  }
  return HPSI_OK;
}

hpsi_status hpsi_apply_h_points(hpsi_hamiltonian *h, const hpsi_batch *psi, hpsi_batch *hpsi, int32_t terms,
                                int32_t set_bc, int32_t points, void *stream) {
  if (!h) return HPSI_ERR_ARG;
  hpsi_status s = check_points(h, terms, points, "hpsi_apply_h_points");
  if (s) return s;
  if (points == 0) return hpsi_apply_h(h, psi, hpsi, terms, set_bc, stream);
  hpsi_mesh *m = h->mesh;
  s = check_batch(m, psi, m->np_part, "hpsi_apply_h_points(psi)");
  if (!s) s = check_batch(m, hpsi, m->np, "hpsi_apply_h_points(hpsi)");
  if (s) return s;
  if (psi->dtype != hpsi->dtype || psi->nst != hpsi->nst || !is_device_ptr(psi->ptr) || !is_device_ptr(hpsi->ptr)) {
    set_error("hpsi_apply_h_points: device batches of one dtype and nst expected");
    return HPSI_ERR_ARG;
  }
  if ((terms & HPSI_TERM_KINETIC) && !h->have_kinetic) {
    set_error("hpsi_apply_h_points: kinetic weights not set");
    return HPSI_ERR_STATE;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (psi->dtype == HPSI_C128)
    return run_pass<double>(h, terms, load_map(h, set_bc), static_cast<const double *>(psi->ptr), psi->ld,
                            static_cast<double *>(hpsi->ptr), hpsi->ld, psi->ld, PASS_APPLY, nullptr, 0, 0.0, 0.0,
                            nullptr, nullptr, st, nullptr, points);
  return run_pass<float>(h, terms, load_map(h, set_bc), static_cast<const float *>(psi->ptr), psi->ld,
                         static_cast<float *>(hpsi->ptr), hpsi->ld, psi->ld, PASS_APPLY, nullptr, 0, 0.0, 0.0,
                         nullptr, nullptr, st, nullptr, points);
}

hpsi_status hpsi_apply_h_horner_points(hpsi_hamiltonian *h, const hpsi_batch *psi, const hpsi_batch *psi0,
                                       hpsi_batch *out, double a_re, double a_im, int32_t terms, int32_t set_bc,
                                       int32_t points, void *stream) {
  if (!h) return HPSI_ERR_ARG;
  hpsi_status s = check_points(h, terms, points, "hpsi_apply_h_horner_points");
  if (s) return s;
  if (points == 0) return hpsi_apply_h_horner(h, psi, psi0, out, a_re, a_im, terms, set_bc, stream);
  hpsi_mesh *m = h->mesh;
  s = check_batch(m, psi, m->np_part, "hpsi_apply_h_horner_points(psi)");
  if (!s) s = check_batch(m, psi0, m->np, "hpsi_apply_h_horner_points(psi0)");
  if (!s) s = check_batch(m, out, m->np, "hpsi_apply_h_horner_points(out)");
  if (s) return s;
  if (psi->dtype != out->dtype || psi0->dtype != out->dtype || psi->ld != out->ld || psi0->ld != out->ld ||
      psi->nst != out->nst || psi0->nst != out->nst || !is_device_ptr(psi->ptr) || !is_device_ptr(psi0->ptr) ||
      !is_device_ptr(out->ptr) || psi->ptr == out->ptr) {
    set_error("hpsi_apply_h_horner_points: device batches of one dtype, ld and nst, out not psi");
    return HPSI_ERR_ARG;
  }
  if ((terms & HPSI_TERM_KINETIC) && !h->have_kinetic) {
    set_error("hpsi_apply_h_horner_points: kinetic weights not set");
    return HPSI_ERR_STATE;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const long long ld = out->ld;
  if (out->dtype == HPSI_C128)
    return run_pass<double>(h, terms, load_map(h, set_bc), static_cast<const double *>(psi->ptr), ld,
                            static_cast<double *>(out->ptr), ld, ld, PASS_HORNER,
                            static_cast<const double *>(psi0->ptr), ld, a_re, a_im, nullptr, nullptr, st, nullptr,
                            points);
  return run_pass<float>(h, terms, load_map(h, set_bc), static_cast<const float *>(psi->ptr), ld,
                         static_cast<float *>(out->ptr), ld, ld, PASS_HORNER, static_cast<const float *>(psi0->ptr),
                         ld, a_re, a_im, nullptr, nullptr, st, nullptr, points);
}

hpsi_status hpsi_hamiltonian_status(hpsi_hamiltonian *h, int32_t *status) {
  if (!h || !status) return HPSI_ERR_ARG;
  *status = HPSI_OK;
  if (!h->d_err) return HPSI_OK;
  int v = 0;
  HPSI_TRY_CUDA(cudaMemcpy(&v, h->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  HPSI_TRY_CUDA(cudaMemset(h->d_err, 0, sizeof(int)));
  *status = v;
  return HPSI_OK;
}

}  // extern "C"
