// Exact discrete adjoint of the Taylor propagator (FP64).
//
// Forward:  psi_{n+1} = T_n psi_n,  T_n = sum_{k=0..K} c_k H_n^k,  c_k = (-i dt)^k / k!,
//           H_n = H_0 + eps_n Z (Z = pol.r, a diagonal operator).
// Objective J = sum_i |<phi_i|psi_i(N)>|^2  (target_j1_groundstate-style,
//           src/opt_control/target_groundstate_inc.F90:83-152),
//           lambda_N = phi <phi|psi(N)> (target_chi_groundstate).
// Backward: lambda_n = T_n^dagger lambda_{n+1} = sum_k conj(c_k) H_n^k lambda_{n+1}
//           (H_n Hermitian, so T_n(dt)^dagger = T_n(-dt)).
// Gradients (vector-Jacobian products), with dT/dtheta = sum_k c_k sum_{j+m=k-1} H^j (dH) H^m:
//   dJ/d eps_n = 2 Re sum_{j+m<=K-1} c_{j+m+1} <H^j lambda_{n+1}| Z |H^m psi_n>,
//   dJ/d v(r)  = 2 Re sum_n sum_{j+m<=K-1} c_{j+m+1} dV sum_i conj(H^j lambda_{n+1})_i(r) (H^m psi_n)_i(r).
// The reference's opt_control uses the continuous-adjoint form
// d_n = 2 Im <chi|Z|psi> dt (calculate_g / update_field,
// src/opt_control/propagation.F90:932-998, 1016-1103); it is the leading
// (j = m = 0) term above and is returned beside the exact gradient.  psi_n is
// recomputed from checkpoints stored every `ckpt` steps, one segment at a time.
#include <cmath>
#include <complex>
#include <cstring>
#include <string>
#include <vector>

#include "api_internal.cuh"
#include "reduce.cuh"

namespace hpsi {

template <typename T>
hpsi_status taylor_dev(hpsi_hamiltonian *h, T *psi, long long ld, int nst, double dt_re, double dt_im, int order,
                       double *obs_dev, cudaStream_t st);
template <typename T>
hpsi_status apply_h_dev(hpsi_hamiltonian *h, const T *psi, long long ld, T *hpsi, long long ldo, int terms,
                        int set_bc, cudaStream_t st);

namespace {

constexpr int KMAX = 8;

struct AdjCoef {
  double cre[KMAX + 1], cim[KMAX + 1];  // c_k
  int K;
};

struct AdjPtrs {
  const double2 *L[KMAX + 1];  // H^k lambda_{n+1}
  const double2 *P[KMAX];      // H^m psi_n
};

// One warp per mesh row.  For each state: s = sum_j conj(L_j) Phi_j with
// Phi_j = sum_{m <= K-1-j} c_{j+m+1} P_m; lambda_new = sum_k conj(c_k) L_k
// written over L_0.  w(r) = sum_i Re s_i; gv[r] += 2 dV w; the eps gradient
// partial of the block += 2 dV z(r) w, and the same for the leading term.
__global__ void __launch_bounds__(256) adj_accumulate_kernel(double2 *L0, const AdjPtrs ptr, long long ld, int nst,
                                                             int np, const AdjCoef c, const double *zrow, double dv,
                                                             double *gv, double *geps_partial,
                                                             double *gcont_partial) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int rows_per_block = blockDim.x >> 5;
  Kahan ke = {0, 0}, kc = {0, 0};
  for (long long r = (long long)blockIdx.x * rows_per_block + warp; r < np;
       r += (long long)gridDim.x * rows_per_block) {
    double wr = 0.0, wc = 0.0;
    for (int i = lane; i < nst; i += 32) {
      const long long o = r * ld + i;
      double2 Pm[KMAX], Lk[KMAX + 1];
      for (int m = 0; m < c.K; ++m) Pm[m] = ptr.P[m][o];
      for (int k = 0; k <= c.K; ++k) Lk[k] = ptr.L[k][o];
      double sre = 0.0;
      for (int j = 0; j < c.K; ++j) {
        double pre = 0.0, pim = 0.0;  // Phi_j
        for (int m = 0; m + j <= c.K - 1; ++m) {
          const double ar = c.cre[j + m + 1], ai = c.cim[j + m + 1];
          pre += ar * Pm[m].x - ai * Pm[m].y;
          pim += ar * Pm[m].y + ai * Pm[m].x;
        }
        sre += Lk[j].x * pre + Lk[j].y * pim;  // Re(conj(L_j) Phi_j)
      }
      wr += sre;
      // leading term only: Re(c_1 conj(L_0) P_0) (the continuous-adjoint form)
      const double cr = Lk[0].x * Pm[0].x + Lk[0].y * Pm[0].y, ci = Lk[0].x * Pm[0].y - Lk[0].y * Pm[0].x;
      wc += c.cre[1] * cr - c.cim[1] * ci;
      double nre = 0.0, nim = 0.0;  // lambda_new = sum conj(c_k) L_k
      for (int k = 0; k <= c.K; ++k) {
        const double ar = c.cre[k], ai = -c.cim[k];
        nre += ar * Lk[k].x - ai * Lk[k].y;
        nim += ar * Lk[k].y + ai * Lk[k].x;
      }
      L0[o] = make_double2(nre, nim);
    }
    for (int off = 16; off > 0; off >>= 1) {
      wr += __shfl_xor_sync(0xffffffffu, wr, off);
      wc += __shfl_xor_sync(0xffffffffu, wc, off);
    }
    if (lane == 0) {
      gv[r] += 2.0 * dv * wr;
      kadd(ke, 2.0 * dv * wr * zrow[r]);
      kadd(kc, 2.0 * dv * wc * zrow[r]);
    }
  }
  __shared__ double red[8][4];
  if (lane == 0) {
    red[warp][0] = ke.s;
    red[warp][1] = ke.c;
    red[warp][2] = kc.s;
    red[warp][3] = kc.c;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    Kahan a = {0, 0}, b = {0, 0};
    for (int w = 0; w < rows_per_block; ++w) {
      kadd(a, red[w][0]);
      a.c += red[w][1];
      kadd(b, red[w][2]);
      b.c += red[w][3];
    }
    geps_partial[2 * blockIdx.x] = a.s;
    geps_partial[2 * blockIdx.x + 1] = a.c;
    gcont_partial[2 * blockIdx.x] = b.s;
    gcont_partial[2 * blockIdx.x + 1] = b.c;
  }
}

__global__ void adj_sum_partials(const double *part, int n, double *out) {
  if (threadIdx.x || blockIdx.x) return;
  Kahan a = {0, 0};
  for (int i = 0; i < n; ++i) {
    kadd(a, part[2 * i]);
    a.c += part[2 * i + 1];
  }
  *out = a.s + a.c;
}

// lambda_i = phi_i * ov_i (ov = per-state complex overlap <phi_i|psi_i>, interleaved)
__global__ void adj_init_lambda(double2 *lam, const double2 *phi, long long ldphi, long long ld, int nst, int np,
                                const double *ov) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= (long long)np * ld) return;
  const long long r = i / ld;
  const int s = int(i % ld);
  if (s >= nst) {
    lam[i] = make_double2(0.0, 0.0);
    return;
  }
  const double2 f = phi[r * ldphi + s];
  const double ar = ov[2 * s], ai = ov[2 * s + 1];
  lam[i] = make_double2(f.x * ar - f.y * ai, f.x * ai + f.y * ar);
}

}  // namespace

struct AdjointRun {
  hpsi_hamiltonian *h;
  long long ld;
  int nst, np, K;
  double dt, pol[3];
  cudaStream_t st;
};

static hpsi_status adj_apply(const AdjointRun &R, double eps, const double2 *in, double2 *out) {
  for (int a = 0; a < 3; ++a) R.h->fld[a] = R.pol[a] * eps;
  return apply_h_dev<double>(R.h, reinterpret_cast<const double *>(in), R.ld, reinterpret_cast<double *>(out), R.ld,
                             HPSI_TERM_ALL, 1, R.st);
}

static hpsi_status adj_step_forward(const AdjointRun &R, double eps, double2 *psi) {
  for (int a = 0; a < 3; ++a) R.h->fld[a] = R.pol[a] * eps;
  return taylor_dev<double>(R.h, reinterpret_cast<double *>(psi), R.ld, R.nst, R.dt, 0.0, R.K, nullptr, R.st);
}

}  // namespace hpsi

using namespace hpsi;

extern "C" hpsi_status hpsi_adjoint_gradient(hpsi_hamiltonian *h, const hpsi_batch *psi0, const hpsi_batch *targets,
                                             int32_t nsteps, double dt, int32_t order, const double *eps,
                                             const double pol[3], int32_t ckpt, double *J_out, double *grad_eps,
                                             double *grad_v, double *grad_eps_cont, void *stream) {
  if (!h || !psi0 || !targets || nsteps < 1 || !(dt > 0.0) || order < 1 || order > KMAX || !eps || !pol ||
      ckpt < 1) {
    set_error("hpsi_adjoint_gradient: bad argument");
    return HPSI_ERR_ARG;
  }
  hpsi_mesh *m = h->mesh;
  if (psi0->dtype != HPSI_C128 || targets->dtype != HPSI_C128 || psi0->nst != targets->nst ||
      psi0->npts < m->np || targets->npts < m->np || psi0->ld < psi0->nst || targets->ld < targets->nst ||
      !is_device_ptr(psi0->ptr) || !is_device_ptr(targets->ptr)) {
    set_error("hpsi_adjoint_gradient: psi0 and targets must be matching complex128 device batches");
    return HPSI_ERR_ARG;
  }
  if (!h->have_kinetic) {
    set_error("hpsi_adjoint_gradient: kinetic weights not set");
    return HPSI_ERR_STATE;
  }
  for (int n = 0; n < nsteps; ++n)
    if (!std::isfinite(eps[n])) {
      set_error("hpsi_adjoint_gradient: non-finite control amplitude");
      return HPSI_ERR_NONFINITE;
    }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  AdjointRun R{h, psi0->ld, psi0->nst, m->np, order, dt, {pol[0], pol[1], pol[2]}, st};
  const size_t batch = size_t(m->np) * R.ld;  // complex numbers of one batch
  const int nseg = (nsteps + ckpt - 1) / ckpt;
  const int seglen = std::min(ckpt, nsteps);
  const int nblk = 296;
  // complex buffers: checkpoints nseg, segment seglen, L[K+1], P[1..K-1]
  const size_t ncplx = batch * (size_t(nseg) + seglen + (order + 1) + order);
  // doubles: zrow np, gv np, 2 partials 2*nblk each, ov 2*ld, ov partial 4*ld, geps nsteps, gcont nsteps
  const size_t ndbl = size_t(m->np) * 2 + 4 * size_t(nblk) + 6 * size_t(R.ld) + 2 * size_t(nsteps) + 8;
  hpsi_status s = h->adjbuf.ensure(ncplx * sizeof(double2) + ndbl * sizeof(double));
  if (s) return s;
  double2 *ckp = static_cast<double2 *>(h->adjbuf.ptr);
  double2 *seg = ckp + batch * nseg;
  double2 *Lb = seg + batch * seglen;
  double2 *Pb = Lb + batch * (order + 1);
  double *zrow = reinterpret_cast<double *>(Pb + batch * order);
  double *gv = zrow + m->np;
  double *part = gv + m->np;
  double *partc = part + 2 * nblk;
  double *ov = partc + 2 * nblk;     // 2*ld
  double *ovpart = ov + 2 * R.ld;    // 4*ld (state_sum partial of one block)
  double *geps = ovpart + 4 * R.ld;  // nsteps
  double *gcont = geps + nsteps;     // nsteps

  // Z = pol . r per inner row
  {
    std::vector<double> z(m->np);
    for (int r = 0; r < m->np; ++r) {
      const int c = m->cell_of_row_h[r];
      const int x = c % m->box.NX, y = (c / m->box.NX) % m->box.NY, zz = c / (m->box.NX * m->box.NY);
      z[r] = pol[0] * (x + m->box.lo[0]) * m->box.h[0] + pol[1] * (y + m->box.lo[1]) * m->box.h[1] +
             pol[2] * (zz + m->box.lo[2]) * m->box.h[2];
    }
    HPSI_TRY_CUDA(cudaMemcpyAsync(zrow, z.data(), z.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    HPSI_TRY_CUDA(cudaStreamSynchronize(st));
  }
  HPSI_TRY_CUDA(cudaMemsetAsync(gv, 0, size_t(m->np) * sizeof(double), st));
  const double dv = m->box.h[0] * m->box.h[1] * m->box.h[2];
  const double save_fld[3] = {h->fld[0], h->fld[1], h->fld[2]};
  auto fail = [&](hpsi_status e) {
    for (int a = 0; a < 3; ++a) h->fld[a] = save_fld[a];
    return e;
  };

  // ---- forward with checkpoints -------------------------------------------------
  double2 *cur = seg;
  HPSI_TRY_CUDA(cudaMemcpy2DAsync(cur, R.ld * sizeof(double2), psi0->ptr, psi0->ld * sizeof(double2),
                                  R.ld * sizeof(double2), m->np, cudaMemcpyDeviceToDevice, st));
  for (int n = 0; n < nsteps; ++n) {
    if (n % ckpt == 0)
      HPSI_TRY_CUDA(cudaMemcpyAsync(ckp + batch * (n / ckpt), cur, batch * sizeof(double2), cudaMemcpyDeviceToDevice,
                                    st));
    s = adj_step_forward(R, eps[n], cur);
    if (s) return fail(s);
  }
  // J and lambda_N
  s = launch_state_sum<double>(1, static_cast<const double *>(targets->ptr), targets->ld,
                               reinterpret_cast<const double *>(cur), R.ld, m->np, R.nst, ovpart, 1, dv, 0, ov, st);
  if (s) return fail(s);
  std::vector<double> ovh(2 * size_t(R.nst));
  HPSI_TRY_CUDA(cudaMemcpyAsync(ovh.data(), ov, ovh.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
  HPSI_TRY_CUDA(cudaStreamSynchronize(st));
  double J = 0.0;
  for (int i = 0; i < R.nst; ++i) J += ovh[2 * i] * ovh[2 * i] + ovh[2 * i + 1] * ovh[2 * i + 1];
  if (J_out) *J_out = J;
  {
    const long long n = (long long)batch;
    adj_init_lambda<<<unsigned((n + 255) / 256), 256, 0, st>>>(Lb, static_cast<const double2 *>(targets->ptr),
                                                                targets->ld, R.ld, R.nst, m->np, ov);
    HPSI_CHECK_LAUNCH();
  }
  // coefficients c_k = (-i dt)^k / k!
  AdjCoef coef;
  coef.K = order;
  {
    std::complex<double> ck(1.0, 0.0);
    for (int k = 0; k <= order; ++k) {
      if (k > 0) ck *= std::complex<double>(0.0, -dt) / double(k);
      coef.cre[k] = ck.real();
      coef.cim[k] = ck.imag();
    }
  }
  AdjPtrs ptr;
  std::memset(&ptr, 0, sizeof(ptr));
  for (int k = 0; k <= order; ++k) ptr.L[k] = Lb + batch * k;
  for (int k = 1; k < order; ++k) ptr.P[k] = Pb + batch * k;

  // ---- backward, one checkpoint segment at a time --------------------------------
  for (int sgi = nseg - 1; sgi >= 0; --sgi) {
    const int n0 = sgi * ckpt, n1 = std::min(nsteps, n0 + ckpt);
    HPSI_TRY_CUDA(cudaMemcpyAsync(seg, ckp + batch * sgi, batch * sizeof(double2), cudaMemcpyDeviceToDevice, st));
    for (int n = n0; n + 1 < n1; ++n) {  // psi_n for n in [n0, n1) into segment slots
      double2 *nxt = seg + batch * (n - n0 + 1);
      HPSI_TRY_CUDA(
          cudaMemcpyAsync(nxt, seg + batch * (n - n0), batch * sizeof(double2), cudaMemcpyDeviceToDevice, st));
      s = adj_step_forward(R, eps[n], nxt);
      if (s) return fail(s);
    }
    for (int n = n1 - 1; n >= n0; --n) {
      ptr.P[0] = seg + batch * (n - n0);
      for (int k = 1; k < order && !s; ++k) s = adj_apply(R, eps[n], ptr.P[k - 1], const_cast<double2 *>(ptr.P[k]));
      for (int k = 1; k <= order && !s; ++k)
        s = adj_apply(R, eps[n], ptr.L[k - 1], const_cast<double2 *>(ptr.L[k]));
      if (s) return fail(s);
      adj_accumulate_kernel<<<nblk, 256, 0, st>>>(Lb, ptr, R.ld, R.nst, m->np, coef, zrow, dv, gv, part, partc);
      HPSI_CHECK_LAUNCH();
      adj_sum_partials<<<1, 32, 0, st>>>(part, nblk, geps + n);
      HPSI_CHECK_LAUNCH();
      adj_sum_partials<<<1, 32, 0, st>>>(partc, nblk, gcont + n);
      HPSI_CHECK_LAUNCH();
    }
  }
  if (grad_eps) HPSI_TRY_CUDA(cudaMemcpyAsync(grad_eps, geps, nsteps * sizeof(double), cudaMemcpyDeviceToHost, st));
  if (grad_eps_cont)
    HPSI_TRY_CUDA(cudaMemcpyAsync(grad_eps_cont, gcont, nsteps * sizeof(double), cudaMemcpyDeviceToHost, st));
  if (grad_v) HPSI_TRY_CUDA(cudaMemcpyAsync(grad_v, gv, size_t(m->np) * sizeof(double), cudaMemcpyDeviceToHost, st));
  HPSI_TRY_CUDA(cudaStreamSynchronize(st));
  for (int a = 0; a < 3; ++a) h->fld[a] = save_fld[a];
  return HPSI_OK;
}
