// Lanczos exponential of a batch (exponential_lanczos_batch,
// src/electrons/exponential.F90:766-901): per state, the Krylov space of
// H is built from psi with classical Gram-Schmidt against the last two
// vectors (X(mesh_batch_orthogonalization), src/grid/mesh_batch_inc.F90:1168-1274,
// the reference's default CGS scheme); the first column of exp(-i dt H_m)
// of the small projected matrix comes from the eigen-decomposition of its
// upper triangle on the host (the reference's Hermitian zlalg_exp path), and
// the iteration stops when every state's error estimate
// |h(m+1, m) expo(m, 1)| (Saad 1992, Er2) is below tol or the space breaks
// down.  psi <- beta sum_j expo(j, 1) v_j.  FP64 batches on the device.
#include <cmath>
#include <complex>
#include <algorithm>
#include <cstring>
#include <thread>
#include <vector>

#include "api_internal.cuh"
#include "reduce.cuh"

namespace hpsi {

template <typename T>
hpsi_status apply_h_dev(hpsi_hamiltonian *h, const T *psi, long long ld, T *hpsi, long long ldo, int terms,
                        int set_bc, cudaStream_t st);

namespace {

using cplx = std::complex<double>;

// The Krylov vectors are kept unnormalised: u_0 = psi (in place, never
// copied), v_j = u_j / sc_j with sc_j = ||u_j|| (1 where the norm is below
// the breakdown threshold, as the reference leaves such vectors unscaled).
// Per iteration two passes over the batch besides H u:
//   lz_sum_kernel<1>: raw overlaps <u_a|w>, <u_b|w> of w = H u_{m-1} with the
//                     last two vectors (one read of w, u_a, u_b);
//   lz_sum_kernel<2>: u_m = w / sc_{m-1} - sum_j raw_j / (sc_j^2 sc_{m-1}) u_j
//                     written over w, with ||u_m||^2 accumulated on the way.
// Sums: per-thread and per-block compensated, partial[nblk][nst][4], then
// lz_finalize in a fixed block order (deterministic).
//
// small device arrays (doubles):
//   raw[nst][4]        dv <u_a|w>, dv <u_b|w>  (re, im each)
//   nrm[K + 1][nst]    ||u_j||
//   sc[K + 1][nst]     scale of v_j
struct LzCoef {
  const double *raw;  // [nst][4]
  const double *sc_prev, *sc_a, *sc_b;  // [nst] each (sc_b null when absent)
};

template <int MODE>
__global__ void __launch_bounds__(256) lz_sum_kernel(double2 *__restrict__ w, const double2 *__restrict__ a,
                                                    const double2 *__restrict__ b, long long ld,
                                                    int np, int nst, LzCoef cf, double *partial) {
  const int rem = nst - int(blockIdx.y) * 256;
  const int SW = rem >= 256 ? 256 : rem;
  const int G = 256 / SW;
  const int t = threadIdx.x;
  const int sl = t % SW, g = t / SW;
  const int s = blockIdx.y * 256 + sl;
  const long long rows_per = (np + gridDim.x - 1) / gridDim.x;
  const long long r0 = blockIdx.x * rows_per;
  const long long r1 = min((long long)np, r0 + rows_per);
  Kahan k[4] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
  if (g < G && s < nst) {
    double f = 1.0;
    double2 ca = make_double2(0.0, 0.0), cb = make_double2(0.0, 0.0);
    if (MODE == 2) {
      const double *o = cf.raw + 4 * (long long)s;
      const double sp = cf.sc_prev[s], sa = cf.sc_a[s];
      f = 1.0 / sp;
      const double qa = 1.0 / (sa * sa * sp);
      ca = make_double2(o[0] * qa, o[1] * qa);
      if (b) {
        const double sb = cf.sc_b[s], qb = 1.0 / (sb * sb * sp);
        cb = make_double2(o[2] * qb, o[3] * qb);
      }
    }
#pragma unroll 4
    for (long long r = r0 + g; r < r1; r += G) {
      const long long o = r * ld + s;
      const double2 x = w[o];
      if (MODE == 0) {
        kadd(k[0], x.x * x.x + x.y * x.y);
      } else if (MODE == 1) {
        const double2 ya = a[o];
        kadd(k[0], ya.x * x.x + ya.y * x.y);
        kadd(k[1], ya.x * x.y - ya.y * x.x);
        if (b) {
          const double2 yb = b[o];
          kadd(k[2], yb.x * x.x + yb.y * x.y);
          kadd(k[3], yb.x * x.y - yb.y * x.x);
        }
      } else {
        const double2 ya = a[o];
        double ux = f * x.x - (ca.x * ya.x - ca.y * ya.y);
        double uy = f * x.y - (ca.x * ya.y + ca.y * ya.x);
        if (b) {
          const double2 yb = b[o];
          ux -= cb.x * yb.x - cb.y * yb.y;
          uy -= cb.x * yb.y + cb.y * yb.x;
        }
        w[o] = make_double2(ux, uy);
        kadd(k[0], ux * ux + uy * uy);
      }
    }
  }
  constexpr int NQ = MODE == 1 ? 4 : 1;
  __shared__ double red[256][NQ];
  for (int q = 0; q < NQ; ++q) red[t][q] = k[q].s + k[q].c;
  __syncthreads();
  if (t < SW && s < nst) {
    Kahan acc[NQ];
    for (int q = 0; q < NQ; ++q) acc[q] = {0, 0};
    for (int gg = 0; gg < G; ++gg)
      for (int q = 0; q < NQ; ++q) kadd(acc[q], red[gg * SW + t][q]);
    double *o = partial + ((long long)blockIdx.x * nst + s) * 4;
    for (int q = 0; q < NQ; ++q) o[q] = acc[q].s + acc[q].c;
  }
}

// Sum partial[nblk][nst][4] over blocks: one CTA of 256 threads per state,
// thread t takes blocks t, t + 256, ... (compensated), then a fixed-order
// tree in shared memory (deterministic).  nq == 4: raw[s][q] = dv * sum.
// nq == 1: nrm[s] = sqrt(dv * sum), sc[s] = nrm >= 1e4 eps ? nrm : 1.
__global__ void __launch_bounds__(256) lz_finalize(const double *partial, int nblk, int nst, int nq, double dv,
                                                  double *raw, double *nrm, double *sc) {
  const int s = blockIdx.x, t = threadIdx.x;
  Kahan acc[4] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
  for (int b = t; b < nblk; b += 256) {
    const double *p = partial + ((long long)b * nst + s) * 4;
    for (int q = 0; q < nq; ++q) kadd(acc[q], p[q]);
  }
  __shared__ double red[4][256];
  for (int q = 0; q < 4; ++q) red[q][t] = acc[q].s + acc[q].c;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (t < w)
      for (int q = 0; q < nq; ++q) red[q][t] += red[q][t + w];
    __syncthreads();
  }
  if (t == 0) {
    if (nq == 4) {
      for (int q = 0; q < 4; ++q) raw[4 * s + q] = dv * red[q][0];
    } else {
      const double n = sqrt(dv * red[0][0]);
      nrm[s] = n;
      sc[s] = n >= 1e4 * 2.220446049250313e-16 ? n : 1.0;
    }
  }
}

// psi[p][s] = c[0][s] psi[p][s] + sum_{j>=1} c[j][s] U_j[p][s]   (U_j = U + (j-1) vstride)
__global__ void lz_combine(double2 *psi, const double2 *U, long long vstride, int m, long long ld, long long n,
                           int nst, const double2 *c) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int s = int(i % nst);
    const long long o = (i / nst) * ld + s;
    double2 x = psi[o], a = c[s];
    double re = a.x * x.x - a.y * x.y, im = a.x * x.y + a.y * x.x;
    for (int j = 1; j < m; ++j) {
      x = U[(j - 1) * vstride + o];
      a = c[j * nst + s];
      re += a.x * x.x - a.y * x.y;
      im += a.x * x.y + a.y * x.x;
    }
    psi[o] = make_double2(re, im);
  }
}

// Eigenvalues of a real symmetric tridiagonal matrix (diagonal a, off-diagonal
// b, both length n, b[n-1] unused) by implicit QR steps with the Wilkinson
// shift and Givens bulge chasing, deflating negligible off-diagonals (Golub &
// Van Loan, Matrix Computations, sec. 8.3).  On return a holds the
// eigenvalues; the rotations are recorded in order (plane (k, k+1), cosine,
// sine) instead of accumulated, so that the eigenvector matrix
// Z = R_1^T R_2^T ... R_N^T is applied to one vector in O(N).  False if a block
// needs more than 30 n sweeps.
struct Givens {
  int k;
  double c, s;
};

bool tridiag_eigen(int n, std::vector<double> &a, std::vector<double> &b, std::vector<Givens> &rot) {
  const double eps = 2.220446049250313e-16;
  rot.clear();
  int hi = n - 1, sweeps = 0;
  while (hi > 0) {
    // deflate at the bottom
    if (std::abs(b[hi - 1]) <= eps * (std::abs(a[hi - 1]) + std::abs(a[hi]))) {
      b[hi - 1] = 0.0;
      --hi;
      continue;
    }
    int lo = hi - 1;
    while (lo > 0 && std::abs(b[lo - 1]) > eps * (std::abs(a[lo - 1]) + std::abs(a[lo]))) --lo;
    if (lo > 0) b[lo - 1] = 0.0;
    if (++sweeps > 30 * n) return false;
    // Wilkinson shift from the trailing 2 x 2 block of [lo, hi]
    const double d = 0.5 * (a[hi - 1] - a[hi]), e2 = b[hi - 1] * b[hi - 1];
    const double mu = a[hi] - e2 / (d + std::copysign(std::sqrt(d * d + e2), d == 0.0 ? 1.0 : d));
    double x = a[lo] - mu, z = b[lo];
    double bulge = 0.0;
    for (int k = lo; k < hi; ++k) {
      // rotation R in the (k, k+1) plane with R (x, z)^T = (r, 0)^T; T <- R T R^T
      const double r = std::sqrt(x * x + z * z);  // |x|, |z| far from overflow here
      const double c = r == 0.0 ? 1.0 : x / r, s = r == 0.0 ? 0.0 : -z / r;
      if (k > lo) b[k - 1] = c * b[k - 1] - s * bulge;  // the bulge at (k+1, k-1) is annihilated
      const double ak = a[k], ak1 = a[k + 1], bk = b[k];
      a[k] = c * c * ak - 2.0 * c * s * bk + s * s * ak1;
      a[k + 1] = s * s * ak + 2.0 * c * s * bk + c * c * ak1;
      b[k] = c * s * (ak - ak1) + (c * c - s * s) * bk;
      if (k + 1 < hi) {
        const double bn = b[k + 1];
        bulge = -s * bn;  // new entry at (k+2, k)
        b[k + 1] = c * bn;
        x = b[k];
        z = bulge;
      }
      rot.push_back({k, c, s});
    }
  }
  return true;
}

// First column of exp(-i dt T) for the Hermitian tridiagonal T whose upper
// triangle is (diag re(hd[j]), super hu[j]) -- the part of the projected
// matrix a Hermitian eigensolver reads.  T = D S D^H with D = diag(phase)
// makes S real symmetric with off-diagonals |hu[j]|, so
// exp(-i dt T) e_1 = D Z exp(-i dt L) Z^T e_1.
bool tridiag_exp_col0(int n, const cplx *hd, const cplx *hu, double dt, std::vector<cplx> &col) {
  std::vector<double> a(n), b(n, 0.0), q(n, 0.0);
  std::vector<cplx> ph(n);
  std::vector<Givens> rot;
  rot.reserve(size_t(4) * n * n);
  ph[0] = 1.0;
  for (int j = 0; j < n; ++j) {
    a[j] = hd[j].real();
    if (j + 1 < n) {
      const double m = std::abs(hu[j]);
      b[j] = m;
      ph[j + 1] = m > 0.0 ? ph[j] * std::conj(hu[j]) / m : ph[j];
    }
  }
  if (!tridiag_eigen(n, a, b, rot)) return false;
  // q = Z^T e_1 = R_N ... R_1 e_1
  q[0] = 1.0;
  for (const Givens &g : rot) {
    const double u = q[g.k], v = q[g.k + 1];
    q[g.k] = g.c * u - g.s * v;
    q[g.k + 1] = g.s * u + g.c * v;
  }
  // col = Z (exp(-i dt L) q) = R_1^T (... (R_N^T y))
  col.resize(n);
  for (int k = 0; k < n; ++k) col[k] = std::polar(q[k], -dt * a[k]);
  for (size_t r = rot.size(); r-- > 0;) {
    const Givens &g = rot[r];
    const cplx u = col[g.k], v = col[g.k + 1];
    col[g.k] = g.c * u + g.s * v;
    col[g.k + 1] = -g.s * u + g.c * v;
  }
  for (int r = 0; r < n; ++r) col[r] *= ph[r];
  return true;
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
  // reduction blocks: 8 per SM (1184 on a B200), at least 256 rows each
  const int nblk = int(std::max(1LL, std::min(1184LL, ((long long)np + 255) / 256)));
  // u_1 .. u_K on the device (u_0 is psi itself)
  hpsi_status s = h->lzbuf.ensure(size_t(K) * vstride * sizeof(double2));
  const size_t small = size_t(nblk) * nst * 4 + 4 * size_t(nst) + 2 * size_t(K + 1) * nst + 2 * size_t(K + 1) * nst;
  if (!s) s = h->lzsmall.ensure(small * sizeof(double));
  if (s) return s;
  double2 *U = static_cast<double2 *>(h->lzbuf.ptr);
  double *partial = static_cast<double *>(h->lzsmall.ptr);
  double *raw = partial + size_t(nblk) * nst * 4;  // [nst][4]
  double *nrm = raw + 4 * size_t(nst);              // [K+1][nst]
  double *sc = nrm + size_t(K + 1) * nst;           // [K+1][nst]
  double2 *coef = reinterpret_cast<double2 *>(sc + size_t(K + 1) * nst);  // [K+1][nst]
  double2 *psi_d = static_cast<double2 *>(psi->ptr);
  auto vec = [&](int j) { return j == 0 ? psi_d : U + (j - 1) * vstride; };
  const dim3 rgrid(nblk, (nst + 255) / 256);

  // host copies: norms and scales of every vector, raw overlaps of this iteration
  std::vector<double> hn(size_t(K + 1) * nst), hs(size_t(K + 1) * nst), hraw(4 * size_t(nst));
  auto fetch = [&](int j, bool with_raw) -> hpsi_status {
    HPSI_TRY_CUDA(cudaMemcpyAsync(hn.data() + size_t(j) * nst, nrm + size_t(j) * nst, nst * sizeof(double),
                                  cudaMemcpyDeviceToHost, st));
    if (with_raw)
      HPSI_TRY_CUDA(cudaMemcpyAsync(hraw.data(), raw, hraw.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    HPSI_TRY_CUDA(cudaStreamSynchronize(st));
    for (int i = 0; i < nst; ++i) {
      const double n = hn[size_t(j) * nst + i];
      hs[size_t(j) * nst + i] = n >= 1e4 * 2.220446049250313e-16 ? n : 1.0;
    }
    return HPSI_OK;
  };

  // beta = ||psi||
  LzCoef none{nullptr, nullptr, nullptr, nullptr};
  lz_sum_kernel<0><<<rgrid, 256, 0, st>>>(psi_d, nullptr, nullptr, ld, np, nst, none, partial);
  HPSI_CHECK_LAUNCH();
  lz_finalize<<<nst, 256, 0, st>>>(partial, nblk, nst, 1, dv, nullptr, nrm, sc);
  HPSI_CHECK_LAUNCH();
  s = fetch(0, false);
  if (s) return s;
  bool all_null = true;
  for (int i = 0; i < nst; ++i) all_null = all_null && std::abs(hn[i]) <= 1e-12;
  if (all_null) {
    if (iters_out) *iters_out = 0;
    if (res_out) *res_out = 0.0;
    return HPSI_OK;
  }

  const unsigned hw = std::thread::hardware_concurrency();
  const int hw_threads = int(std::min(16u, std::max(1u, hw)));
  // projected matrices (row-major (K+1) x (K+1) per state), first columns of their exponentials
  std::vector<std::vector<cplx>> H(nst, std::vector<cplx>(size_t(K + 1) * (K + 1), 0.0));
  std::vector<std::vector<cplx>> expo(nst);
  std::vector<double> res(nst, 0.0);
  int iter = 1;
  for (; iter <= K; ++iter) {
    // w = H u_{iter-1} into u_iter's slot, then CGS against v_l-1 .. v_iter-1, l = max(1, iter - 1)
    s = apply_h_dev<double>(h, reinterpret_cast<const double *>(vec(iter - 1)), ld,
                            reinterpret_cast<double *>(vec(iter)), ld, HPSI_TERM_ALL, 1, st);
    if (s) return s;
    const int l = std::max(1, iter - 1);
    const bool two = iter - l == 1;
    const double2 *ua = vec(l - 1), *ub = two ? vec(l) : nullptr;
    lz_sum_kernel<1><<<rgrid, 256, 0, st>>>(vec(iter), ua, ub, ld, np, nst, none, partial);
    HPSI_CHECK_LAUNCH();
    lz_finalize<<<nst, 256, 0, st>>>(partial, nblk, nst, 4, dv, raw, nullptr, nullptr);
    HPSI_CHECK_LAUNCH();
    LzCoef cf{raw, sc + size_t(iter - 1) * nst, sc + size_t(l - 1) * nst, two ? sc + size_t(l) * nst : nullptr};
    lz_sum_kernel<2><<<rgrid, 256, 0, st>>>(vec(iter), ua, ub, ld, np, nst, cf, partial);
    HPSI_CHECK_LAUNCH();
    lz_finalize<<<nst, 256, 0, st>>>(partial, nblk, nst, 1, dv, nullptr, nrm + size_t(iter) * nst,
                                       sc + size_t(iter) * nst);
    HPSI_CHECK_LAUNCH();
    s = fetch(iter, true);
    if (s) return s;
    const double *sp = hs.data() + size_t(iter - 1) * nst;
    std::vector<char> ok(nst, 1);
    auto host_state = [&](int i) {
      // overlaps <v_j | H v_iter-1> = raw_j / (sc_j sc_iter-1)
      for (int j = l; j <= iter; ++j) {
        const double *r = hraw.data() + 4 * size_t(i) + 2 * (j - l);
        H[i][size_t(j - 1) * (K + 1) + (iter - 1)] = cplx(r[0], r[1]) / (hs[size_t(j - 1) * nst + i] * sp[i]);
      }
      const double ni = hn[size_t(iter) * nst + i];
      H[i][size_t(iter) * (K + 1) + (iter - 1)] = ni;
      // first column of exp(-i dt H_iter), H_iter the leading iter x iter block
      std::vector<cplx> hd(iter), hu(iter);
      for (int a = 0; a < iter; ++a) {
        hd[a] = H[i][size_t(a) * (K + 1) + a];
        if (a + 1 < iter) hu[a] = H[i][size_t(a) * (K + 1) + a + 1];
      }
      ok[i] = tridiag_exp_col0(iter, hd.data(), hu.data(), dt, expo[i]);
      res[i] = ok[i] ? ni * std::abs(expo[i][iter - 1]) : 0.0;
    };
    // the small eigenproblems are independent: spread them over host threads
    // when there is enough work (about 20 ns per state per iter^2)
    const int nthr = int(std::min<long long>({(long long)hw_threads, (long long)nst / 4,
                                              (long long)nst * iter * iter / 4000 + 1}));
    if (nthr > 1) {
      std::vector<std::thread> pool;
      for (int t = 0; t < nthr; ++t)
        pool.emplace_back([&, t] {
          for (int i = t; i < nst; i += nthr) host_state(i);
        });
      for (auto &th : pool) th.join();
    } else {
      for (int i = 0; i < nst; ++i) host_state(i);
    }
    bool breakdown = true;
    double worst = 0.0;
    for (int i = 0; i < nst; ++i) {
      if (!ok[i]) {
        set_error("hpsi_lanczos_step: eigensolver of the projected matrix did not converge");
        return HPSI_ERR_NONFINITE;
      }
      worst = std::max(worst, res[i]);
      breakdown = breakdown && hn[size_t(iter) * nst + i] < 1e4 * 2.220446049250313e-16;
    }
    if (breakdown) break;  // happy breakdown: the space is invariant
    if (iter > 3 && worst < tol) break;
  }
  const int mdim = std::min(iter, K);
  // psi = beta sum_j expo(j, 1) v_j = sum_j beta expo(j, 1) / sc_j u_j
  std::vector<cplx> cc(size_t(mdim) * nst);
  double worst = 0.0;
  for (int i = 0; i < nst; ++i) {
    worst = std::max(worst, res[i]);
    for (int j = 0; j < mdim; ++j) cc[size_t(j) * nst + i] = hn[i] * expo[i][j] / hs[size_t(j) * nst + i];
  }
  HPSI_TRY_CUDA(cudaMemcpyAsync(coef, cc.data(), cc.size() * sizeof(double2), cudaMemcpyHostToDevice, st));
  lz_combine<<<grid_for(nel), 256, 0, st>>>(psi_d, U, vstride, mdim, ld, nel, nst, coef);
  HPSI_CHECK_LAUNCH();
  HPSI_TRY_CUDA(cudaStreamSynchronize(st));
  if (iters_out) *iters_out = mdim;
  if (res_out) *res_out = worst;  // > tol: not converged (the reference only warns)
  return HPSI_OK;
}
