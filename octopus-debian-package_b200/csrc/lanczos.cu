// Lanczos exponential of a batch (exponential_lanczos_batch,
// src/electrons/exponential.F90:766-901): per state, the Krylov space of
// H is built from psi with classical Gram-Schmidt against the last two
// vectors (X(mesh_batch_orthogonalization), src/grid/mesh_batch_inc.F90:1168-1274,
// the reference's default CGS scheme); the small projected matrix is
// exponentiated on the host (exp(-i dt H_m) by scaling and squaring of its
// Taylor series), and the iteration stops when every state's error estimate
// |h(m+1, m) expo(m, 1)| (Saad 1992, Er2) is below tol or the space breaks
// down.  psi <- beta sum_j expo(j, 1) v_j.  FP64 batches on the device.
#include <cmath>
#include <complex>
#include <cstring>
#include <vector>

#include "api_internal.cuh"
#include "reduce.cuh"

namespace hpsi {

template <typename T>
hpsi_status apply_h_dev(hpsi_hamiltonian *h, const T *psi, long long ld, T *hpsi, long long ldo, int terms,
                        int set_bc, cudaStream_t st);
int reduce_blocks(int np);

namespace {

using cplx = std::complex<double>;

// v[p][s] *= c[s]
__global__ void lz_scale(double2 *v, long long ld, long long n, int nst, const double2 *c) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int s = int(i % nst);
    const long long p = i / nst;
    const double2 x = v[p * ld + s], a = c[s];
    v[p * ld + s] = make_double2(a.x * x.x - a.y * x.y, a.x * x.y + a.y * x.x);
  }
}

// w[p][s] -= ca[s] a[p][s] + cb[s] b[p][s]   (b may be null)
__global__ void lz_sub(double2 *w, const double2 *a, const double2 *b, long long ld, long long n, int nst,
                       const double2 *ca, const double2 *cb) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int s = int(i % nst);
    const long long p = i / nst, o = p * ld + s;
    double2 y = w[o];
    const double2 x = a[o], c = ca[s];
    y.x -= c.x * x.x - c.y * x.y;
    y.y -= c.x * x.y + c.y * x.x;
    if (b) {
      const double2 z = b[o], d = cb[s];
      y.x -= d.x * z.x - d.y * z.y;
      y.y -= d.x * z.y + d.y * z.x;
    }
    w[o] = y;
  }
}

// psi[p][s] = sum_j c[j][s] V_j[p][s]
__global__ void lz_combine(double2 *psi, long long ldp, const double2 *V, long long vstride, int m, long long ld,
                           long long n, int nst, const double2 *c) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int s = int(i % nst);
    const long long p = i / nst;
    double re = 0.0, im = 0.0;
    for (int j = 0; j < m; ++j) {
      const double2 x = V[j * vstride + p * ld + s], a = c[j * nst + s];
      re += a.x * x.x - a.y * x.y;
      im += a.x * x.y + a.y * x.x;
    }
    psi[p * ldp + s] = make_double2(re, im);
  }
}

// exp(A) for a small complex matrix (row-major m x m): scaling and squaring of
// the Taylor series (terms until they fall below 1e-18 of the running sum).
std::vector<cplx> small_expm(const std::vector<cplx> &A, int m) {
  double nrm = 0.0;
  for (int j = 0; j < m; ++j) {
    double c = 0.0;
    for (int i = 0; i < m; ++i) c += std::abs(A[i * m + j]);
    nrm = std::max(nrm, c);
  }
  int sq = 0;
  while (nrm > 0.5) {
    nrm *= 0.5;
    ++sq;
  }
  const double f = std::ldexp(1.0, -sq);
  std::vector<cplx> B(A), E(m * m, 0.0), term(m * m, 0.0), tmp(m * m);
  for (auto &x : B) x *= f;
  for (int i = 0; i < m; ++i) E[i * m + i] = term[i * m + i] = 1.0;
  for (int k = 1; k <= 40; ++k) {
    for (int i = 0; i < m; ++i)
      for (int j = 0; j < m; ++j) {
        cplx acc = 0.0;
        for (int l = 0; l < m; ++l) acc += term[i * m + l] * B[l * m + j];
        tmp[i * m + j] = acc / double(k);
      }
    term.swap(tmp);
    double tn = 0.0, en = 0.0;
    for (int i = 0; i < m * m; ++i) {
      E[i] += term[i];
      tn = std::max(tn, std::abs(term[i]));
      en = std::max(en, std::abs(E[i]));
    }
    if (tn <= 1e-18 * en) break;
  }
  for (int r = 0; r < sq; ++r) {
    for (int i = 0; i < m; ++i)
      for (int j = 0; j < m; ++j) {
        cplx acc = 0.0;
        for (int l = 0; l < m; ++l) acc += E[i * m + l] * E[l * m + j];
        tmp[i * m + j] = acc;
      }
    E.swap(tmp);
  }
  return E;
}

unsigned grid_for(long long n) { return unsigned(std::min<long long>((n + 255) / 256, 148 * 32)); }

}  // namespace

}  // namespace hpsi

using namespace hpsi;

extern "C" hpsi_status hpsi_lanczos_step(hpsi_hamiltonian *h, hpsi_batch *psi, double dt, int32_t max_order,
                                         double tol, int32_t *iters_out, double *res_out, void *stream) {
  if (!h || !psi || !(dt > 0.0) || max_order < 2 || max_order > 64 || !(tol > 0.0)) {
    set_error("hpsi_lanczos_step: bad argument");
    return HPSI_ERR_ARG;
  }
  if (!h->have_kinetic) {
    set_error("hpsi_lanczos_step: kinetic weights not set");
    return HPSI_ERR_STATE;
  }
  hpsi_mesh *m = h->mesh;
  if (psi->dtype != HPSI_C128) {
    set_error("hpsi_lanczos_step: complex128 batches only");
    return HPSI_ERR_UNSUPPORTED;
  }
  if (!psi->ptr || psi->npts < m->np || psi->nst < 1 || psi->ld < psi->nst || !is_device_ptr(psi->ptr)) {
    set_error("hpsi_lanczos_step: device batch with at least np points expected");
    return HPSI_ERR_ARG;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int nst = psi->nst, np = m->np, K = max_order;
  const long long ld = psi->ld;
  const long long vstride = (long long)np * ld;  // complex numbers per Krylov vector
  const long long nel = (long long)np * nst;
  const double dv = m->box.h[0] * m->box.h[1] * m->box.h[2];
  const int nblk = reduce_blocks(np);
  hpsi_status s = h->lzbuf.ensure(size_t(K + 1) * vstride * sizeof(double2));
  if (!s) s = h->lzsmall.ensure((size_t(nblk) * nst * 4 + 2 * nst + 2 * size_t(K + 1) * nst) * sizeof(double));
  if (s) return s;
  double2 *V = static_cast<double2 *>(h->lzbuf.ptr);
  double *partial = static_cast<double *>(h->lzsmall.ptr);
  double *red = partial + size_t(nblk) * nst * 4;         // [nst][2]
  double2 *coef = reinterpret_cast<double2 *>(red + 2 * nst);  // [(K+1)][nst]
  double2 *psi_d = static_cast<double2 *>(psi->ptr);
  auto vec = [&](int j) { return V + j * vstride; };

  // host reductions: <a|b> per state (dv-scaled), or norms
  std::vector<double> hred(2 * size_t(nst));
  auto dot = [&](const double2 *a, const double2 *b, std::vector<cplx> &out) -> hpsi_status {
    hpsi_status r = launch_state_sum<double>(1, reinterpret_cast<const double *>(a), ld,
                                             reinterpret_cast<const double *>(b), ld, np, nst, partial, nblk, dv, 0,
                                             red, st);
    if (r) return r;
    HPSI_TRY_CUDA(cudaMemcpyAsync(hred.data(), red, hred.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    HPSI_TRY_CUDA(cudaStreamSynchronize(st));
    out.resize(nst);
    for (int i = 0; i < nst; ++i) out[i] = cplx(hred[2 * i], hred[2 * i + 1]);
    return HPSI_OK;
  };
  auto norm = [&](const double2 *a, std::vector<double> &out) -> hpsi_status {
    hpsi_status r = launch_state_sum<double>(0, reinterpret_cast<const double *>(a), ld, nullptr, 0, np, nst, partial,
                                             nblk, dv, 1, red, st);
    if (r) return r;
    HPSI_TRY_CUDA(cudaMemcpyAsync(hred.data(), red, hred.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    HPSI_TRY_CUDA(cudaStreamSynchronize(st));
    out.resize(nst);
    for (int i = 0; i < nst; ++i) out[i] = hred[2 * i];
    return HPSI_OK;
  };
  auto put = [&](double2 *dst, const std::vector<cplx> &c) -> hpsi_status {
    HPSI_TRY_CUDA(cudaMemcpyAsync(dst, c.data(), c.size() * sizeof(double2), cudaMemcpyHostToDevice, st));
    HPSI_TRY_CUDA(cudaStreamSynchronize(st));  // the host vector is reused
    return HPSI_OK;
  };

  // v_1 = psi / beta
  HPSI_TRY_CUDA(cudaMemcpyAsync(vec(0), psi_d, size_t(vstride) * sizeof(double2), cudaMemcpyDeviceToDevice, st));
  std::vector<double> beta;
  s = norm(vec(0), beta);
  if (s) return s;
  bool all_null = true;
  for (double b : beta) all_null = all_null && std::abs(b) <= 1e-12;
  if (all_null) {
    if (iters_out) *iters_out = 0;
    if (res_out) *res_out = 0.0;
    return HPSI_OK;
  }
  std::vector<cplx> c(nst);
  for (int i = 0; i < nst; ++i) c[i] = beta[i] > 0.0 ? 1.0 / beta[i] : 1.0;
  s = put(coef, c);
  if (s) return s;
  lz_scale<<<grid_for(nel), 256, 0, st>>>(vec(0), ld, nel, nst, coef);
  HPSI_CHECK_LAUNCH();

  // projected matrices (row-major (K+1) x (K+1) per state) and the exponentials
  std::vector<std::vector<cplx>> H(nst, std::vector<cplx>(size_t(K + 1) * (K + 1), 0.0));
  std::vector<std::vector<cplx>> expo(nst);
  std::vector<double> res(nst, 0.0);
  int iter = 1;
  for (; iter <= K; ++iter) {
    // v_iter+1 = H v_iter, then CGS against v_l .. v_iter, l = max(1, iter - 1)
    s = apply_h_dev<double>(h, reinterpret_cast<const double *>(vec(iter - 1)), ld,
                            reinterpret_cast<double *>(vec(iter)), ld, HPSI_TERM_ALL, 1, st);
    if (s) return s;
    const int l = std::max(1, iter - 1);
    std::vector<std::vector<cplx>> ov;
    for (int j = l; j <= iter; ++j) {
      std::vector<cplx> o;
      s = dot(vec(j - 1), vec(iter), o);
      if (s) return s;
      ov.push_back(o);
    }
    for (int i = 0; i < nst; ++i)
      for (int j = l; j <= iter; ++j) H[i][size_t(j - 1) * (K + 1) + (iter - 1)] = ov[j - l][i];
    // w -= sum_j ov_j v_j
    std::vector<cplx> c1 = ov[0], c2 = ov.size() > 1 ? ov[1] : std::vector<cplx>();
    s = put(coef, c1);
    if (!s && !c2.empty()) s = put(coef + nst, c2);
    if (s) return s;
    lz_sub<<<grid_for(nel), 256, 0, st>>>(vec(iter), vec(l - 1), c2.empty() ? nullptr : vec(l), ld, nel, nst, coef,
                                          coef + nst);
    HPSI_CHECK_LAUNCH();
    std::vector<double> nrm;
    s = norm(vec(iter), nrm);
    if (s) return s;
    bool breakdown = true;
    double worst = 0.0;
    for (int i = 0; i < nst; ++i) {
      H[i][size_t(iter) * (K + 1) + (iter - 1)] = nrm[i];
      // exp(-i dt H_iter) of the leading iter x iter block
      std::vector<cplx> A(size_t(iter) * iter);
      for (int a = 0; a < iter; ++a)
        for (int b = 0; b < iter; ++b) A[a * iter + b] = cplx(0.0, -dt) * H[i][size_t(a) * (K + 1) + b];
      expo[i] = small_expm(A, iter);
      res[i] = std::abs(nrm[i]) * std::abs(expo[i][size_t(iter - 1) * iter]);
      worst = std::max(worst, res[i]);
      breakdown = breakdown && std::abs(nrm[i]) < 1e4 * 2.220446049250313e-16;
    }
    if (breakdown) break;  // happy breakdown: the space is invariant
    for (int i = 0; i < nst; ++i) c[i] = std::abs(nrm[i]) >= 1e4 * 2.220446049250313e-16 ? 1.0 / std::abs(nrm[i]) : 1.0;
    s = put(coef, c);
    if (s) return s;
    lz_scale<<<grid_for(nel), 256, 0, st>>>(vec(iter), ld, nel, nst, coef);
    HPSI_CHECK_LAUNCH();
    if (iter > 3 && worst < tol) break;
  }
  const int mdim = std::min(iter, K);
  // psi = beta sum_j expo(j, 1) v_j
  std::vector<cplx> cc(size_t(mdim) * nst);
  double worst = 0.0;
  for (int i = 0; i < nst; ++i) {
    worst = std::max(worst, res[i]);
    for (int j = 0; j < mdim; ++j) cc[size_t(j) * nst + i] = beta[i] * expo[i][size_t(j) * mdim];
  }
  HPSI_TRY_CUDA(cudaMemcpyAsync(coef, cc.data(), cc.size() * sizeof(double2), cudaMemcpyHostToDevice, st));
  lz_combine<<<grid_for(nel), 256, 0, st>>>(psi_d, psi->ld, V, vstride, mdim, ld, nel, nst, coef);
  HPSI_CHECK_LAUNCH();
  HPSI_TRY_CUDA(cudaStreamSynchronize(st));
  if (iters_out) *iters_out = mdim;
  if (res_out) *res_out = worst;  // > tol: not converged (the reference only warns)
  return HPSI_OK;
}
