// Many independent systems per launch, and the pass autotuner.
//
// A group holds the Hamiltonians of independent systems (uneven meshes and
// state counts).  One Taylor step runs, per Horner pass, the KB bra of every
// system, then ONE persistent launch of the fused stencil pass over a work
// list of (system, tile column + z block, state chunk) units sorted by cost,
// then the KB ket of every system; the whole step can be captured in a CUDA
// graph and replayed.  There is no reference counterpart to the grouping: the
// reference loops over state blocks on the host
// (propagation_ops_elec_fuse_density_exp_apply, src/td/propagation_ops_elec.F90:261-333),
// one kernel launch per block and sub-step.
//
// The autotuner times the candidate pass shapes (state chunk width, z block
// depth) of a Hamiltonian on scratch batches and keeps the fastest.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "api_internal.cuh"
#include "projector.cuh"
#include "stencil_blk.cuh"

namespace hpsi {

PassShape pass_shape(const hpsi_hamiltonian *h, int dtype, long long ld);
PassShape default_shape(int dtype, long long ld);
int pass_sc(int dtype, long long ld);
int choose_zb(const hpsi_mesh *m, int chunks, int ty);
hpsi_status mesh_items(hpsi_mesh *m, int zb, int ty, const int4 **items, int *nitems);
PassShape blk_shape(int dtype);
const int *load_map(const hpsi_hamiltonian *h, int set_bc);
hpsi_status prepare_taylor_workspaces(hpsi_hamiltonian *h, long long ld, size_t elem, bool obs);
template <typename T>
hpsi_status build_pass_args(hpsi_hamiltonian *h, int terms, const int *src_map, const T *in, long long in_ld, T *out,
                            long long out_ld, long long ld, int mode, const T *psi0, long long psi0_ld, double a_re,
                            double a_im, const PassShape &shape, PassArgs &a);
template <typename T>
hpsi_status run_bra(hpsi_hamiltonian *h, const T *psi, long long ld, T *proj, cudaStream_t st);
template <typename T>
hpsi_status run_ket(hpsi_hamiltonian *h, const T *proj, long long ld, int nst, T *out, long long out_ld, int mode,
                    double a_re, double a_im, const T *psi0, long long psi0_ld, double *obs, cudaStream_t st,
                    double *rho_ket = nullptr, const double *rho_w = nullptr, int row_blocks = 0);
template <typename T>
hpsi_status launch_pass(PassArgs a, const PassShape &shape, cudaStream_t st);
template <typename T>
hpsi_status launch_pass_any(const PassArgs &a, const PassShape &shape, long long in_rows, cudaStream_t st);

namespace {
template <typename T>
__global__ void copy_rows_group_kernel(const T *src, T *dst, long long ld, long long n) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) dst[i] = src[i];
}
}  // namespace

}  // namespace hpsi

struct hpsi_group {
  std::vector<hpsi_hamiltonian *> hams;
  // launch sub-groups of at most GROUP_MAX systems: [first, end) and units
  struct Launch {
    int first = 0, end = 0;
    int4 *d_units = nullptr;
    int nunits = 0;
  };
  std::vector<Launch> launches;
  long long built_ld_sig = -1;  // signature of the batch widths the units were built for
  int built_dtype = -1, sc = 0;
  bool blk = false;             // every width fits the blocked pass's chunk
  std::vector<hpsi::PassShape> shapes;
  int *d_counter = nullptr;     // one counter per launch sub-group
  cudaStream_t cap = nullptr;
  cudaEvent_t ev = nullptr;
  // side streams: the per-system KB bras and kets run concurrently (forked
  // from and joined back to the step's stream; branches of the captured graph)
  std::vector<cudaStream_t> side;
  std::vector<cudaEvent_t> join;
  cudaEvent_t fork = nullptr;
  int num_sms = 148;
};

namespace hpsi {

static void group_free_units(hpsi_group *g) {
  for (auto &l : g->launches) dev_free(l.d_units);
  g->launches.clear();
}

// Build the per-launch unit lists for batches of widths ld[s].
static hpsi_status group_build(hpsi_group *g, int dtype, const std::vector<long long> &ld) {
  long long sig = dtype;
  for (long long x : ld) sig = sig * 1315423911LL + x;
  if (sig == g->built_ld_sig && !g->launches.empty()) return HPSI_OK;
  group_free_units(g);
  const int n = int(g->hams.size());
  g->shapes.assign(n, PassShape{});
  // the blocked pass when every width is a multiple of its chunk
  const PassShape bs = blk_shape(dtype);
  g->blk = true;
  for (int s = 0; s < n; ++s) g->blk = g->blk && ld[s] % bs.sc == 0;
  if (g->blk) {
    for (int s = 0; s < n; ++s) g->shapes[s] = default_shape(dtype, ld[s]);
    for (int s = 0; s < n; ++s)
      if (!g->shapes[s].blk || g->shapes[s].rx != g->shapes[0].rx || g->shapes[s].ry != g->shapes[0].ry ||
          g->shapes[s].cplx != g->shapes[0].cplx || g->shapes[s].unroll != g->shapes[0].unroll ||
          g->shapes[s].sc != g->shapes[0].sc || g->shapes[s].ty != g->shapes[0].ty || ld[s] % g->shapes[s].sc) {
        g->blk = false;
        break;
      }
  }
  // common state chunk: the smallest preferred chunk over the systems
  int sc = g->blk ? g->shapes[0].sc : (dtype == HPSI_C128 ? 4 : 8);
  for (int s = 0; s < n && !g->blk; ++s) {
    PassShape sh = pass_shape(g->hams[s], dtype, ld[s]);
    sc = std::min(sc, sh.blk ? (dtype == HPSI_C128 ? 4 : 8) : sh.sc);
    g->shapes[s] = sh;
  }
  for (int s = 0; s < n && !g->blk; ++s) {
    if (ld[s] % sc) {
      set_error("hpsi_group: batch width incompatible with the common state chunk");
      return HPSI_ERR_UNSUPPORTED;
    }
    g->shapes[s].sc = sc;
    g->shapes[s].ry = dtype == HPSI_C128 ? 2 : 4;
    g->shapes[s].tx = g->shapes[s].ty = 16;
    g->shapes[s].blk = 0;  // the one-complex-per-thread pass
    g->shapes[s].zb = 0;
  }
  g->sc = sc;
  // z block depth: whole tile columns (each item re-reads a 4-plane halo above
  // and below its block, 8 planes per item) unless the group as a whole would
  // then give fewer than four waves of units, in which case every system takes
  // the depth it would take alone
  {
    long long units_full = 0;
    for (int s = 0; s < n; ++s) {
      const int ty = g->blk ? g->shapes[s].ty : 16;
      const auto &tz = ty == 8 ? g->hams[s]->mesh->tile_z8 : g->hams[s]->mesh->tile_z;
      long long t = 0;
      for (auto &c : tz) t += c.y >= 0;
      units_full += t * (ld[s] / sc);
    }
    if (units_full >= 4LL * g->num_sms)
      for (int s = 0; s < n; ++s)
        if (g->shapes[s].zb <= 0) g->shapes[s].zb = 1 << 20;
  }
  for (int first = 0; first < n; first += GROUP_MAX) {
    hpsi_group::Launch L;
    L.first = first;
    L.end = std::min(n, first + GROUP_MAX);
    std::vector<std::pair<long long, int4>> units;
    for (int s = L.first; s < L.end; ++s) {
      hpsi_hamiltonian *h = g->hams[s];
      const int chunks = int(ld[s] / sc);
      const int ty = g->blk ? g->shapes[s].ty : 16;
      const int zb = g->shapes[s].zb > 0 ? g->shapes[s].zb : choose_zb(h->mesh, chunks, ty);
      g->shapes[s].zb = zb;
      const int4 *items;
      int nitems = 0;
      hpsi_status st = mesh_items(h->mesh, zb, ty, &items, &nitems);
      if (st) return st;
      // the items live on the device; recompute their z extents on the host for the cost
      std::vector<int4> hi(nitems);
      if (nitems) HPSI_TRY_CUDA(cudaMemcpy(hi.data(), items, nitems * sizeof(int4), cudaMemcpyDeviceToHost));
      for (int i = 0; i < nitems; ++i)
        for (int c = 0; c < chunks; ++c)
          units.push_back({(long long)(hi[i].w - hi[i].z + 8), make_int4(s - L.first, i, c, 0)});
    }
    std::stable_sort(units.begin(), units.end(), [](const auto &a, const auto &b) { return a.first > b.first; });
    std::vector<int4> u(units.size());
    for (size_t i = 0; i < units.size(); ++i) u[i] = units[i].second;
    hpsi_status st = dev_alloc(reinterpret_cast<void **>(&L.d_units), std::max<size_t>(1, u.size()) * sizeof(int4));
    if (st) return st;
    if (!u.empty()) HPSI_TRY_CUDA(cudaMemcpy(L.d_units, u.data(), u.size() * sizeof(int4), cudaMemcpyHostToDevice));
    L.nunits = int(u.size());
    g->launches.push_back(L);
  }
  g->built_ld_sig = sig;
  g->built_dtype = dtype;
  return HPSI_OK;
}

template <typename T>
static hpsi_status group_step(hpsi_group *g, const std::vector<T *> &psi, const std::vector<long long> &ld,
                              const std::vector<int> &nst, double dt, int order, cudaStream_t st) {
  const int n = int(g->hams.size());
  const int ns = int(g->side.size());
  auto fork = [&]() -> hpsi_status {
    HPSI_TRY_CUDA(cudaEventRecord(g->fork, st));
    for (int i = 0; i < ns; ++i) HPSI_TRY_CUDA(cudaStreamWaitEvent(g->side[i], g->fork, 0));
    return HPSI_OK;
  };
  auto join = [&]() -> hpsi_status {
    for (int i = 0; i < ns; ++i) {
      HPSI_TRY_CUDA(cudaEventRecord(g->join[i], g->side[i]));
      HPSI_TRY_CUDA(cudaStreamWaitEvent(st, g->join[i], 0));
    }
    return HPSI_OK;
  };
  auto sst = [&](int s) { return ns ? g->side[s % ns] : st; };
  std::vector<const T *> in(psi.begin(), psi.end());
  for (int k = order; k >= 1; --k) {
    const double are = 0.0 / k, aim = -dt / k;  // a_k = -i dt / k (real dt)
    std::vector<T *> out(n);
    hpsi_status r0 = fork();
    if (r0) return r0;
    for (int s = 0; s < n; ++s) {
      hpsi_hamiltonian *h = g->hams[s];
      T *u0 = static_cast<T *>(h->u[0].ptr), *u1 = static_cast<T *>(h->u[1].ptr);
      out[s] = (k == 1 && order > 1) ? psi[s] : ((order - k) % 2 == 0 ? u0 : u1);
      if (h->nmat > 0) {
        hpsi_status r = run_bra<T>(h, in[s], ld[s], static_cast<T *>(h->projbuf.ptr), sst(s));
        if (r) return r;
      }
    }
    r0 = join();
    if (r0) return r0;
    for (size_t li = 0; li < g->launches.size(); ++li) {
      const auto &L = g->launches[li];
      GroupArgs ga;
      std::memset(&ga, 0, sizeof(ga));
      for (int s = L.first; s < L.end; ++s) {
        hpsi_hamiltonian *h = g->hams[s];
        hpsi_status r = build_pass_args<T>(h, HPSI_TERM_ALL, load_map(h, 1), in[s], ld[s], out[s], ld[s], ld[s],
                                           PASS_HORNER, psi[s], ld[s], are, aim, g->shapes[s], ga.sys[s - L.first]);
        if (r) return r;
      }
      ga.units = L.d_units;
      ga.nunits = L.nunits;
      ga.counter = g->d_counter + li;
      HPSI_TRY_CUDA(cudaMemsetAsync(ga.counter, 0, sizeof(int), st));
      ProfScope prof(sizeof(T) == 8 ? "group_pass_fp64" : "group_pass_fp32", st);
      const PassShape &s0 = g->shapes[L.first];
      hpsi_status r = g->blk ? launch_pass_blk_group<T>(ga, s0, g->num_sms, st)
                             : launch_pass_group<T>(ga, g->sc, g->num_sms, st);
      if (r) return r;
    }
    r0 = fork();
    if (r0) return r0;
    for (int s = 0; s < n; ++s) {
      hpsi_hamiltonian *h = g->hams[s];
      if (h->nmat > 0) {
        // the kets of the systems run side by side: each takes at most 256 CTA
        // rows (1024 when a ket has the GPU to itself); measured on 64 systems,
        // 4 Taylor steps: 24.16 -> 23.50 ms (FP64), 16.45 -> 16.00 ms (FP32)
        hpsi_status r = run_ket<T>(h, static_cast<const T *>(h->projbuf.ptr), ld[s], int(ld[s]), out[s], ld[s],
                                   PASS_HORNER, are, aim, psi[s], ld[s], nullptr, sst(s), nullptr, nullptr, 256);
        if (r) return r;
      }
    }
    r0 = join();
    if (r0) return r0;
    for (int s = 0; s < n; ++s) in[s] = out[s];
  }
  if (order == 1)
    for (int s = 0; s < n; ++s) {
      const long long cnt = (long long)g->hams[s]->mesh->np * ld[s] * 2;
      copy_rows_group_kernel<T><<<unsigned((cnt + 255) / 256), 256, 0, st>>>(in[s], psi[s], ld[s], cnt);
      HPSI_CHECK_LAUNCH();
    }
  (void)nst;
  return HPSI_OK;
}

template <typename T>
static hpsi_status group_run(hpsi_group *g, hpsi_batch *b, int nsteps, double dt, int order, bool graph,
                             cudaStream_t st) {
  const int n = int(g->hams.size());
  std::vector<T *> psi(n);
  std::vector<long long> ld(n);
  std::vector<int> nst(n);
  for (int s = 0; s < n; ++s) {
    psi[s] = static_cast<T *>(b[s].ptr);
    ld[s] = b[s].ld;
    nst[s] = b[s].nst;
  }
  hpsi_status r = group_build(g, b[0].dtype, ld);
  if (r) return r;
  if (!g->fork) {
    constexpr int NSIDE = 8;
    HPSI_TRY_CUDA(cudaEventCreateWithFlags(&g->fork, cudaEventDisableTiming));
    g->side.resize(NSIDE);
    g->join.resize(NSIDE);
    for (int i = 0; i < NSIDE; ++i) {
      HPSI_TRY_CUDA(cudaStreamCreateWithFlags(&g->side[i], cudaStreamNonBlocking));
      HPSI_TRY_CUDA(cudaEventCreateWithFlags(&g->join[i], cudaEventDisableTiming));
    }
  }
  for (int s = 0; s < n; ++s) {
    r = prepare_taylor_workspaces(g->hams[s], ld[s], sizeof(T), false);
    if (r) return r;
  }
  if (!graph) {
    for (int i = 0; !r && i < nsteps; ++i) r = group_step<T>(g, psi, ld, nst, dt, order, st);
    return r;
  }
  if (!g->cap) {
    HPSI_TRY_CUDA(cudaStreamCreateWithFlags(&g->cap, cudaStreamNonBlocking));
    HPSI_TRY_CUDA(cudaEventCreateWithFlags(&g->ev, cudaEventDisableTiming));
  }
  HPSI_TRY_CUDA(cudaEventRecord(g->ev, st));
  HPSI_TRY_CUDA(cudaStreamWaitEvent(g->cap, g->ev, 0));
  cudaGraph_t graph_h = nullptr;
  cudaGraphExec_t ge = nullptr;
  HPSI_TRY_CUDA(cudaStreamBeginCapture(g->cap, cudaStreamCaptureModeThreadLocal));
  r = group_step<T>(g, psi, ld, nst, dt, order, g->cap);
  cudaError_t e = cudaStreamEndCapture(g->cap, &graph_h);
  if (!r && e != cudaSuccess) {
    set_error(std::string("hpsi_group_taylor_steps: capture: ") + cudaGetErrorString(e));
    r = HPSI_ERR_CUDA;
  }
  if (!r && cudaGraphInstantiate(&ge, graph_h, 0) != cudaSuccess) {
    set_error("hpsi_group_taylor_steps: cudaGraphInstantiate failed");
    r = HPSI_ERR_CUDA;
  }
  for (int i = 0; !r && i < nsteps; ++i) {
    g_launches.fetch_add(1, std::memory_order_relaxed);
    if (cudaGraphLaunch(ge, g->cap) != cudaSuccess) {
      set_error("hpsi_group_taylor_steps: cudaGraphLaunch failed");
      r = HPSI_ERR_CUDA;
    }
  }
  if (ge) cudaGraphExecDestroy(ge);
  if (graph_h) cudaGraphDestroy(graph_h);
  cudaEventRecord(g->ev, g->cap);
  cudaStreamWaitEvent(st, g->ev, 0);
  return r;
}

// ---------------------------------------------------------------------------
// autotuner: time the candidate shapes of the apply pass on scratch batches
template <typename T>
static hpsi_status autotune_t(hpsi_hamiltonian *h, int dtype, long long ld, cudaStream_t st) {
  hpsi_mesh *m = h->mesh;
  const size_t esz = 2 * sizeof(T);
  void *in = nullptr, *out = nullptr;
  hpsi_status r = dev_alloc(&in, size_t(m->np_part) * ld * esz);
  if (!r) r = dev_alloc(&out, size_t(m->np) * ld * esz);
  if (r) {
    dev_free(in);
    return r;
  }
  cudaMemsetAsync(in, 0, size_t(m->np_part) * ld * esz, st);
  std::vector<PassShape> cands;
  const int maxsc = dtype == HPSI_C128 ? 4 : 8;
  const int ry = dtype == HPSI_C128 ? 2 : 4;
  for (int sc = maxsc; sc >= 1 && sc >= maxsc / 2; sc >>= 1) {
    if (ld % sc) continue;
    for (int zb : {0, 16, 24, 32, 48, 64, 96, 1 << 20}) cands.push_back(PassShape{sc, 16, 16, ry, zb});
  }
  // blocked pass: the instantiated cell blocks x z block depths
  const PassShape b0 = blk_shape(dtype);
  if (ld % (b0.sc / 2) == 0) {
    std::vector<PassShape> blocks;
    if (ld % b0.sc == 0) blocks.push_back(b0);
    PassShape b1 = b0, b2 = b0;
    if (dtype == HPSI_C128) {
      b1.unroll = 3;  // real lanes, groups of 3 planes
      b2.cplx = 1;    // complex states, groups of 9
    } else {
      b1.unroll = 3;  // complex states, groups of 3
      b2.cplx = 0;    // real lanes 2 x 4, groups of 1
      b2.ry = 4;
      b2.unroll = 1;
    }
    if (ld % b0.sc == 0) {
      blocks.push_back(b1);
      blocks.push_back(b2);
    }
    {
      PassShape b3 = b0;  // 64-byte chunks, 16 x 16 tiles, 1 x 4 cells
      b3.sc = b0.sc / 2;
      b3.ty = 16;
      b3.rx = 1;
      b3.ry = 4;
      b3.cplx = dtype == HPSI_C128 ? 0 : 1;
      b3.unroll = 9;
      blocks.push_back(b3);
      PassShape b4 = b3;  // 64-byte chunks, 16 x 8 tiles, 256 threads, two CTAs per SM
      b4.ty = 8;
      blocks.push_back(b4);
    }
    if (ld % b0.sc == 0) {
      PassShape bt = b0;  // the default block with the TMA fill of contiguous halo runs
      bt.tma = 1;
      blocks.push_back(bt);
      PassShape bm = b0;  // the default block with the mbarrier hand-over of the stages
      bm.mb = 1;
      blocks.push_back(bm);
    }
    for (const auto &b : blocks)
      for (int zb : {0, 16, 32, 48, 64, 1 << 20}) {
        PassShape c = b;
        c.zb = zb;
        cands.push_back(c);
      }
  }
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  double best = 1e30;
  PassShape best_shape = default_shape(dtype, ld);
  for (const auto &sh0 : cands) {
    PassArgs a;
    PassShape sh = sh0;
    r = build_pass_args<T>(h, HPSI_TERM_KINETIC | HPSI_TERM_LOCAL_POTENTIAL, load_map(h, 1),
                           static_cast<const T *>(in), ld, static_cast<T *>(out), ld, ld, PASS_APPLY, nullptr, 0,
                           0.0, 0.0, sh, a);
    if (!r && sh.blk) r = prepare_tma(h, load_map(h, 1), m->np_part, sh, a);
    if (r) break;
    if (sh0.tma && !sh.tma) continue;  // no TMA table for this load map
    for (int i = 0; i < 2 && !r; ++i) r = launch_pass_any<T>(a, sh, m->np, st);
    cudaEventRecord(e0, st);
    const int reps = 5;
    for (int i = 0; i < reps && !r; ++i) r = launch_pass_any<T>(a, sh, m->np, st);
    cudaEventRecord(e1, st);
    if (r) break;
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms / reps < best) {
      best = ms / reps;
      best_shape = sh;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamSynchronize(st);
  dev_free(in);
  dev_free(out);
  if (r) return r;
  auto &t = h->tuned[dtype == HPSI_C128 ? 0 : 1];
  t.ld = ld;
  t.shape = best_shape;
  t.ms = best;
  return HPSI_OK;
}

}  // namespace hpsi

using namespace hpsi;

extern "C" {

hpsi_status hpsi_group_create(int32_t nsys, hpsi_hamiltonian *const *hams, hpsi_group **out) {
  if (nsys < 1 || !hams || !out) return HPSI_ERR_ARG;
  hpsi_group *g = new hpsi_group();
  for (int s = 0; s < nsys; ++s) {
    if (!hams[s] || !hams[s]->have_kinetic) {
      delete g;
      set_error("hpsi_group_create: every Hamiltonian needs its kinetic weights");
      return HPSI_ERR_STATE;
    }
    g->hams.push_back(hams[s]);
  }
  g->num_sms = hams[0]->mesh->num_sms;
  const int nl = (nsys + GROUP_MAX - 1) / GROUP_MAX;
  hpsi_status s = dev_alloc(reinterpret_cast<void **>(&g->d_counter), nl * sizeof(int));
  if (s) {
    delete g;
    return s;
  }
  *out = g;
  return HPSI_OK;
}

hpsi_status hpsi_group_destroy(hpsi_group *g) {
  if (!g) return HPSI_OK;
  group_free_units(g);
  dev_free(g->d_counter);
  if (g->cap) cudaStreamDestroy(g->cap);
  if (g->ev) cudaEventDestroy(g->ev);
  for (auto s : g->side) cudaStreamDestroy(s);
  for (auto e : g->join) cudaEventDestroy(e);
  if (g->fork) cudaEventDestroy(g->fork);
  delete g;
  return HPSI_OK;
}

hpsi_status hpsi_group_taylor_steps(hpsi_group *g, hpsi_batch *psis, int32_t nsteps, double dt, int32_t order,
                                    int32_t use_graph, void *stream) {
  if (!g || !psis || nsteps < 0 || !(dt > 0.0) || order < 1 || order > 32) return HPSI_ERR_ARG;
  const int n = int(g->hams.size());
  for (int s = 0; s < n; ++s) {
    const hpsi_batch &b = psis[s];
    if (!b.ptr || b.dtype != psis[0].dtype || b.nst < 1 || b.ld < b.nst || b.npts < g->hams[s]->mesh->np ||
        !is_device_ptr(b.ptr)) {
      set_error("hpsi_group_taylor_steps: batch " + std::to_string(s) + " is not a valid device batch");
      return HPSI_ERR_ARG;
    }
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (psis[0].dtype == HPSI_C128) return group_run<double>(g, psis, nsteps, dt, order, use_graph != 0, st);
  return group_run<float>(g, psis, nsteps, dt, order, use_graph != 0, st);
}

hpsi_status hpsi_autotune(hpsi_hamiltonian *h, int32_t dtype, int64_t ld, int32_t shape_out[4], double *ms_out,
                          void *stream) {
  if (!h || ld < 1 || (dtype != HPSI_C128 && dtype != HPSI_C64)) return HPSI_ERR_ARG;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  hpsi_status r = dtype == HPSI_C128 ? autotune_t<double>(h, dtype, ld, st) : autotune_t<float>(h, dtype, ld, st);
  if (r) return r;
  const auto &t = h->tuned[dtype == HPSI_C128 ? 0 : 1];
  if (shape_out) {
    shape_out[0] = t.shape.sc;
    shape_out[1] = t.shape.ry;
    shape_out[2] = t.shape.zb;
    shape_out[3] = t.shape.ty;
  }
  if (ms_out) *ms_out = t.ms;
  return HPSI_OK;
}

}  // extern "C"
