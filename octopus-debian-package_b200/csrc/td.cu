// Time propagation driver: exponential-midpoint steps with a length-gauge
// laser, per-step FP64 observables, optional CUDA-graph replay.
//
// Reference: td_run (src/td/td.F90:546-631) -> propagator_elec_dt ->
// exponential_midpoint (src/td/propagator_expmid.F90:52-100): H is evaluated at
// t + dt/2 (laser E(t+dt/2) folded into the local potential,
// hamiltonian_elec_update, src/hamiltonian/hamiltonian_elec.F90:1028) and one
// Taylor exponential advances the states.  The observables of each step are
// those of psi(t_n) with H(t_n): the fused first pass measures them with
// H(t_n + dt/2) and the laser difference is removed exactly,
// E(t_n) = E_mid - (eps(t_n + dt/2) - eps(t_n)) * <pol.r>, since H depends on the
// field only through eps * pol.r.
//
// ETRS (td_etrs, src/td/propagator_etrs.F90:70-152, independent particles):
// exp(-i dt/2 H(t_n+1)) exp(-i dt/2 H(t_n)); the observables are measured by
// the first half step, with H(t_n) exactly.
#include <cmath>
#include <cstring>
#include <vector>

#include "api_internal.cuh"
#include "reduce.cuh"

namespace hpsi {

template <typename T>
hpsi_status taylor_dev(hpsi_hamiltonian *h, T *psi, long long ld, int nst, double dt_re, double dt_im, int order,
                       double *obs_dev, cudaStream_t st);
hpsi_status prepare_taylor_workspaces(hpsi_hamiltonian *h, long long ld, size_t elem, bool obs);

namespace {

// Sums the per-state observables of the current step over the states and
// advances the device step counter and the field amplitude of the next step.
// tables: amp_mid[nsteps+1], amp_n[nsteps+1]; state: {cur_amp, step}.
__global__ void td_step_finalize(const double *obs_state, int nst, const double *amp_mid, const double *amp_n,
                                 double *cur_amp, int *step, double *energy, double *dipole, double *norm2) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int s = *step;
  Kahan e = {0, 0}, n = {0, 0}, d = {0, 0};
  for (int i = 0; i < nst; ++i) {
    kadd(e, obs_state[i]);
    kadd(n, obs_state[nst + i]);
    kadd(d, obs_state[2 * nst + i]);
  }
  const double D = d.s + d.c;
  energy[s] = (e.s + e.c) - (amp_mid[s] - amp_n[s]) * D;
  dipole[s] = D;
  norm2[s] = n.s + n.c;
  *step = s + 1;
  *cur_amp = amp_mid[s + 1];
}

double laser_field(const hpsi_laser &L, double t) {
  // E(t) = E0 sin^2(pi t / T) cos(omega t) on [0, T], zero outside
  if (t < 0.0 || t > L.T || L.T <= 0.0) return 0.0;
  const double s = std::sin(M_PI * t / L.T);
  return L.E0 * s * s * std::cos(L.omega * t);
}

// ETRS: the second half step of step *step runs with the field of t_n+1.
__global__ void td_set_second_half(const double *amp_b, const int *step, double *cur_amp) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *cur_amp = amp_b[*step];
}

}  // namespace

// propagator: 0 exponential midpoint, 1 ETRS
template <typename T>
hpsi_status td_run(hpsi_hamiltonian *h, T *psi, long long ld, int nst, int nsteps, double dt, int order,
                   const hpsi_laser *las, double t0, bool graph, double *e_out, double *d_out, double *n_out,
                   cudaStream_t st, int propagator = 0) {
  // device layout of the driver buffer (doubles):
  // amp_mid[nsteps+1] amp_n[nsteps+1] cur_amp step(int) E[nsteps] D[nsteps] N[nsteps] obs_state[3*nst]
  // amp_b[nsteps+1]
  // (ETRS: amp_mid = amp_n = E(t_n), the first half step; amp_b = E(t_n+1))
  const bool etrs = propagator == 1;
  const size_t nd = 2 * size_t(nsteps + 1) + 2 + 3 * size_t(nsteps) + 3 * size_t(nst) + size_t(nsteps + 1);
  hpsi_status s = h->tdbuf.ensure(nd * sizeof(double));
  if (s) return s;
  double *base = static_cast<double *>(h->tdbuf.ptr);
  double *amp_mid = base, *amp_n = base + (nsteps + 1), *cur_amp = amp_n + (nsteps + 1);
  int *step = reinterpret_cast<int *>(cur_amp + 1);
  double *E = cur_amp + 2, *D = E + nsteps, *N = D + nsteps, *obs_state = N + nsteps;
  double *amp_b = obs_state + 3 * size_t(nst);
  std::vector<double> host(2 * size_t(nsteps + 1) + 2, 0.0), hostb(size_t(nsteps + 1), 0.0);
  const hpsi_laser none = {0.0, 0.0, 0.0, {0.0, 0.0, 1.0}};
  const hpsi_laser &L = las ? *las : none;
  for (int i = 0; i <= nsteps; ++i) {
    host[i] = laser_field(L, t0 + (etrs ? i : i + 0.5) * dt);
    host[nsteps + 1 + i] = laser_field(L, t0 + i * dt);
    hostb[i] = laser_field(L, t0 + (i + 1) * dt);
  }
  host[2 * size_t(nsteps + 1)] = host[0];  // cur_amp
  int zero = 0;
  std::memcpy(&host[2 * size_t(nsteps + 1) + 1], &zero, sizeof(int));
  HPSI_TRY_CUDA(cudaMemcpyAsync(base, host.data(), host.size() * sizeof(double), cudaMemcpyHostToDevice, st));
  if (etrs)
    HPSI_TRY_CUDA(cudaMemcpyAsync(amp_b, hostb.data(), hostb.size() * sizeof(double), cudaMemcpyHostToDevice, st));

  // the field enters the pass as pol * (*cur_amp)
  const double save_fld[3] = {h->fld[0], h->fld[1], h->fld[2]};
  const double save_pol[3] = {h->pol[0], h->pol[1], h->pol[2]};
  const bool save_have = h->have_pol;
  for (int a = 0; a < 3; ++a) {
    h->fld[a] = L.pol[a];
    h->pol[a] = L.pol[a];
  }
  h->have_pol = true;
  h->fld_scale_dev = cur_amp;

  auto one_step = [&]() -> hpsi_status {
    hpsi_status r = taylor_dev<T>(h, psi, ld, nst, etrs ? 0.5 * dt : dt, 0.0, order, obs_state, st);
    if (r) return r;
    if (etrs) {
      td_set_second_half<<<1, 32, 0, st>>>(amp_b, step, cur_amp);
      HPSI_CHECK_LAUNCH();
      r = taylor_dev<T>(h, psi, ld, nst, 0.5 * dt, 0.0, order, nullptr, st);
      if (r) return r;
    }
    td_step_finalize<<<1, 32, 0, st>>>(obs_state, nst, amp_mid, amp_n, cur_amp, step, E, D, N);
    HPSI_CHECK_LAUNCH();
    return HPSI_OK;
  };

  hpsi_status r = prepare_taylor_workspaces(h, ld, sizeof(T), true);
  if (!r && graph && nsteps > 0) {
    // capture and replay on the handle's own stream, ordered after and
    // before the caller's stream with events (the legacy default stream
    // cannot be captured)
    cudaStream_t cap = h->capture_stream;
    if (!cap) {
      HPSI_TRY_CUDA(cudaStreamCreateWithFlags(&h->capture_stream, cudaStreamNonBlocking));
      HPSI_TRY_CUDA(cudaEventCreateWithFlags(&h->capture_event, cudaEventDisableTiming));
      cap = h->capture_stream;
    }
    HPSI_TRY_CUDA(cudaEventRecord(h->capture_event, st));
    HPSI_TRY_CUDA(cudaStreamWaitEvent(cap, h->capture_event, 0));
    const cudaStream_t user = st;
    st = cap;
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ge = nullptr;
    cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
      set_error(std::string("hpsi_td_propagate: cudaStreamBeginCapture: ") + cudaGetErrorString(e));
      r = HPSI_ERR_CUDA;
    } else {
      r = one_step();
      cudaError_t e2 = cudaStreamEndCapture(st, &g);
      if (!r && e2 != cudaSuccess) {
        set_error(std::string("hpsi_td_propagate: cudaStreamEndCapture: ") + cudaGetErrorString(e2));
        r = HPSI_ERR_CUDA;
      }
      if (!r) {
        e2 = cudaGraphInstantiate(&ge, g, 0);
        if (e2 != cudaSuccess) {
          set_error(std::string("hpsi_td_propagate: cudaGraphInstantiate: ") + cudaGetErrorString(e2));
          r = HPSI_ERR_CUDA;
        }
      }
      for (int i = 0; !r && i < nsteps; ++i) {
        e2 = cudaGraphLaunch(ge, st);
        g_launches.fetch_add(1, std::memory_order_relaxed);
        if (e2 != cudaSuccess) {
          set_error(std::string("hpsi_td_propagate: cudaGraphLaunch: ") + cudaGetErrorString(e2));
          r = HPSI_ERR_CUDA;
        }
      }
      if (ge) cudaGraphExecDestroy(ge);
      if (g) cudaGraphDestroy(g);
    }
    cudaEventRecord(h->capture_event, st);
    cudaStreamWaitEvent(user, h->capture_event, 0);
    st = user;
  } else {
    for (int i = 0; !r && i < nsteps; ++i) r = one_step();
  }
  h->fld_scale_dev = nullptr;
  for (int a = 0; a < 3; ++a) {
    h->fld[a] = save_fld[a];
    h->pol[a] = save_pol[a];
  }
  h->have_pol = save_have;
  if (r) return r;
  std::vector<double> out(3 * size_t(nsteps));
  if (nsteps > 0)
    HPSI_TRY_CUDA(cudaMemcpyAsync(out.data(), E, out.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
  HPSI_TRY_CUDA(cudaStreamSynchronize(st));
  bool finite = true;
  for (double x : out) finite = finite && std::isfinite(x);
  if (e_out) std::memcpy(e_out, out.data(), nsteps * sizeof(double));
  if (d_out) std::memcpy(d_out, out.data() + nsteps, nsteps * sizeof(double));
  if (n_out) std::memcpy(n_out, out.data() + 2 * size_t(nsteps), nsteps * sizeof(double));
  if (!finite) {
    set_error("hpsi_td_propagate: non-finite observable");
    return HPSI_ERR_NONFINITE;
  }
  // Taylor has no stability guarantee: flag norm growth (a runaway series)
  if (nsteps > 0 && out[2 * size_t(nsteps)] > 0.0) {
    const double n0 = out[2 * size_t(nsteps)];
    for (int i = 0; i < nsteps; ++i)
      if (out[2 * size_t(nsteps) + i] > n0 * (1.0 + 1e-3)) {
        set_error("hpsi_td_propagate: norm grew by more than 1e-3 at step " + std::to_string(i) +
                  " (Taylor series runaway; reduce dt)");
        return HPSI_ERR_RUNAWAY;
      }
  }
  return HPSI_OK;
}

}  // namespace hpsi

using namespace hpsi;

static hpsi_status td_entry(const char *name, hpsi_hamiltonian *h, hpsi_batch *psi, int32_t nsteps, double dt,
                            int32_t order, const hpsi_laser *laser, double t0, int32_t use_graph, double *energy,
                            double *dipole, double *norm2, void *stream, int propagator) {
  if (!h || !psi || nsteps < 0 || !(dt > 0.0) || order < 1 || order > 32) {
    set_error(std::string(name) + ": bad argument");
    return HPSI_ERR_ARG;
  }
  if (!h->have_kinetic) {
    set_error(std::string(name) + ": kinetic weights not set");
    return HPSI_ERR_STATE;
  }
  if (!psi->ptr || psi->npts < h->mesh->np || psi->nst < 1 || psi->ld < psi->nst || !is_device_ptr(psi->ptr)) {
    set_error(std::string(name) + ": device batch with at least np points expected");
    return HPSI_ERR_ARG;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (psi->dtype == HPSI_C128)
    return td_run<double>(h, static_cast<double *>(psi->ptr), psi->ld, psi->nst, nsteps, dt, order, laser, t0,
                          use_graph != 0, energy, dipole, norm2, st, propagator);
  if (psi->dtype == HPSI_C64)
    return td_run<float>(h, static_cast<float *>(psi->ptr), psi->ld, psi->nst, nsteps, dt, order, laser, t0,
                         use_graph != 0, energy, dipole, norm2, st, propagator);
  set_error(std::string(name) + ": unknown dtype");
  return HPSI_ERR_ARG;
}

extern "C" hpsi_status hpsi_td_propagate(hpsi_hamiltonian *h, hpsi_batch *psi, int32_t nsteps, double dt,
                                         int32_t order, const hpsi_laser *laser, double t0, int32_t use_graph,
                                         double *energy, double *dipole, double *norm2, void *stream) {
  return td_entry("hpsi_td_propagate", h, psi, nsteps, dt, order, laser, t0, use_graph, energy, dipole, norm2,
                  stream, 0);
}

extern "C" hpsi_status hpsi_td_propagate_etrs(hpsi_hamiltonian *h, hpsi_batch *psi, int32_t nsteps, double dt,
                                              int32_t order, const hpsi_laser *laser, double t0,
                                              int32_t use_graph, double *energy, double *dipole, double *norm2,
                                              void *stream) {
  return td_entry("hpsi_td_propagate_etrs", h, psi, nsteps, dt, order, laser, t0, use_graph, energy, dipole, norm2,
                  stream, 1);
}

// exponential_apply_batch with a second output (psib2, deltat2;
// src/electrons/exponential.F90:695-744): psi2 <- exp(-i dt2 H) psi and
// psi <- exp(-i dt H) psi, both by the order-`order` Taylor series of the same
// H.  The reference accumulates both sums from one sequence H^k psi (power
// form: per term one H apply and two axpys); here psi is copied into psi2 and
// each output gets its own Horner sweep.  On an HBM-bound pass the two move
// the same bytes (power form: read H^(k-1) psi, write H^k psi, update psi and
// psi2 = 6 batch passes per term; two Horner chains: 2 x 3), while the Horner
// form needs no extra batch for H^k psi.
extern "C" hpsi_status hpsi_taylor_step_dual(hpsi_hamiltonian *h, hpsi_batch *psi, hpsi_batch *psi2, double dt_re,
                                             double dt_im, double dt2_re, double dt2_im, int32_t order,
                                             void *stream) {
  if (!h || !psi || !psi2 || order < 1 || order > 32 || !std::isfinite(dt_re) || !std::isfinite(dt_im) ||
      !std::isfinite(dt2_re) || !std::isfinite(dt2_im)) {
    set_error("hpsi_taylor_step_dual: bad argument");
    return HPSI_ERR_ARG;
  }
  if (!h->have_kinetic) {
    set_error("hpsi_taylor_step_dual: kinetic weights not set");
    return HPSI_ERR_STATE;
  }
  const int np = h->mesh->np;
  for (const hpsi_batch *b : {static_cast<const hpsi_batch *>(psi), static_cast<const hpsi_batch *>(psi2)})
    if (!b->ptr || b->npts < np || b->nst < 1 || b->ld < b->nst || !is_device_ptr(b->ptr)) {
      set_error("hpsi_taylor_step_dual: device batches with at least np points expected");
      return HPSI_ERR_ARG;
    }
  if (psi->dtype != psi2->dtype || psi->nst != psi2->nst || (psi->dtype != HPSI_C128 && psi->dtype != HPSI_C64) ||
      psi->ptr == psi2->ptr) {
    set_error("hpsi_taylor_step_dual: psi and psi2 must be distinct batches of one dtype and width");
    return HPSI_ERR_ARG;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const size_t esz = psi->dtype == HPSI_C128 ? 16 : 8;
  HPSI_TRY_CUDA(cudaMemcpy2DAsync(psi2->ptr, size_t(psi2->ld) * esz, psi->ptr, size_t(psi->ld) * esz,
                                  size_t(psi->nst) * esz, np, cudaMemcpyDeviceToDevice, st));
  hpsi_status s;
  if (psi->dtype == HPSI_C128) {
    s = taylor_dev<double>(h, static_cast<double *>(psi2->ptr), psi2->ld, psi2->nst, dt2_re, dt2_im, order, nullptr,
                           st);
    if (!s)
      s = taylor_dev<double>(h, static_cast<double *>(psi->ptr), psi->ld, psi->nst, dt_re, dt_im, order, nullptr, st);
  } else {
    s = taylor_dev<float>(h, static_cast<float *>(psi2->ptr), psi2->ld, psi2->nst, dt2_re, dt2_im, order, nullptr,
                          st);
    if (!s)
      s = taylor_dev<float>(h, static_cast<float *>(psi->ptr), psi->ld, psi->nst, dt_re, dt_im, order, nullptr, st);
  }
  return s;
}
