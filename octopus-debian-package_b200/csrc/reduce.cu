// FP64 reductions over a batch: per-state norms and dot products, the
// overlap (Gram) matrix, its Cholesky factor and the triangular update that
// orthonormalises a batch, and the final reduction of the observables the
// stencil pass accumulates.  All sums are compensated (two-sum) and
// deterministic (fixed partial layout, fixed reduction order).
//
// Reference: X(mesh_batch_nrm2) / X(mesh_batch_dotp_vector) /
// X(mesh_batch_dotp_matrix) (src/grid/mesh_batch_inc.F90:20-263, 379-552,
// 970-1167) and the cholesky_serial branch of
// X(states_elec_orthogonalization_full) (src/states/states_elec_calc_inc.F90:66-98).
#include <algorithm>

#include "reduce.cuh"

namespace hpsi {

namespace {

template <typename T>
struct C2;
template <>
struct C2<double> {
  using type = double2;
};
template <>
struct C2<float> {
  using type = float2;
};

// ---------------------------------------------------------------------------
// per-state sums: grid (nblk, ceil(ld/SW)); block 256 = SW states x G row groups
// mode 0: sum |a|^2 -> q0 ; mode 1: sum conj(a) b -> (q0, q1)
template <typename T, int MODE>
__global__ void __launch_bounds__(256) state_sum_kernel(const T *a, long long lda, const T *b, long long ldb,
                                                       int np, int nst, double *partial) {
  using V = typename C2<T>::type;
  const int SW = min(nst - int(blockIdx.y) * 256, 256) > 0 ? min(nst - int(blockIdx.y) * 256, 256) : 1;
  const int G = 256 / SW;
  const int t = threadIdx.x;
  const int sl = t % SW, g = t / SW;
  const int s = blockIdx.y * 256 + sl;
  const long long rows_per = (np + gridDim.x - 1) / gridDim.x;
  const long long r0 = blockIdx.x * rows_per;
  const long long r1 = min((long long)np, r0 + rows_per);
  Kahan k0 = {0, 0}, k1 = {0, 0};
  if (g < G && s < nst) {
    for (long long r = r0 + g; r < r1; r += G) {
      const V x = reinterpret_cast<const V *>(a + r * 2 * lda)[s];
      if (MODE == 0) {
        kadd(k0, double(x.x) * double(x.x) + double(x.y) * double(x.y));
      } else {
        const V y = reinterpret_cast<const V *>(b + r * 2 * ldb)[s];
        kadd(k0, double(x.x) * double(y.x) + double(x.y) * double(y.y));
        kadd(k1, double(x.x) * double(y.y) - double(x.y) * double(y.x));
      }
    }
  }
  __shared__ double red[256][4];
  red[t][0] = k0.s;
  red[t][1] = k0.c;
  red[t][2] = k1.s;
  red[t][3] = k1.c;
  __syncthreads();
  if (t < SW && s < nst) {
    Kahan a0 = {0, 0}, a1 = {0, 0};
    for (int gg = 0; gg < G; ++gg) {
      const int u = gg * SW + t;
      kadd(a0, red[u][0]);
      a0.c += red[u][1];
      kadd(a1, red[u][2]);
      a1.c += red[u][3];
    }
    double *o = partial + ((long long)blockIdx.x * nst + s) * 4;
    o[0] = a0.s;
    o[1] = a0.c;
    o[2] = a1.s;
    o[3] = a1.c;
  }
}

// sum partial[nblk][nst][4] over blocks -> out[nst][2] (times scale)
__global__ void state_sum_finalize(const double *partial, int nblk, int nst, double scale, int sqrt_first,
                                   double *out) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nst) return;
  Kahan a0 = {0, 0}, a1 = {0, 0};
  for (int b = 0; b < nblk; ++b) {
    const double *p = partial + ((long long)b * nst + s) * 4;
    kadd(a0, p[0]);
    a0.c += p[1];
    kadd(a1, p[2]);
    a1.c += p[3];
  }
  double v0 = (a0.s + a0.c) * scale;
  if (sqrt_first) v0 = sqrt(v0);
  out[2 * s] = v0;
  out[2 * s + 1] = (a1.s + a1.c) * scale;
}

// ---------------------------------------------------------------------------
// Gram matrix of the real views: G[u][v] = sum_p Ar[p][u] Br[p][v],
// u, v over 2*nst real lanes.  grid (ceil(n/32), ceil(n/32), splits),
// block (16,16); each thread a 2x2 block.  Partials [splits][n][n].
template <typename T>
__global__ void __launch_bounds__(256) gram_kernel(const T *a, long long lda, const T *b, long long ldb, int np,
                                                  int n, double *partial) {
  __shared__ double sa[32][33];
  __shared__ double sb[32][33];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int t = ty * 16 + tx;
  const int u0 = blockIdx.y * 32, v0 = blockIdx.x * 32;
  const long long per = (np + gridDim.z - 1) / gridDim.z;
  const long long p0 = blockIdx.z * per, p1 = min((long long)np, p0 + per);
  double c[2][2] = {{0, 0}, {0, 0}};
  for (long long pb = p0; pb < p1; pb += 32) {
    for (int i = t; i < 32 * 32; i += 256) {
      const int pp = i / 32, l = i % 32;
      const long long row = pb + pp;
      sa[pp][l] = (row < p1 && u0 + l < n) ? double(a[row * 2 * lda + u0 + l]) : 0.0;
      sb[pp][l] = (row < p1 && v0 + l < n) ? double(b[row * 2 * ldb + v0 + l]) : 0.0;
    }
    __syncthreads();
#pragma unroll 8
    for (int pp = 0; pp < 32; ++pp) {
      const double a0 = sa[pp][ty * 2], a1 = sa[pp][ty * 2 + 1];
      const double b0 = sb[pp][tx * 2], b1 = sb[pp][tx * 2 + 1];
      c[0][0] = fma(a0, b0, c[0][0]);
      c[0][1] = fma(a0, b1, c[0][1]);
      c[1][0] = fma(a1, b0, c[1][0]);
      c[1][1] = fma(a1, b1, c[1][1]);
    }
    __syncthreads();
  }
  double *o = partial + (long long)blockIdx.z * n * n;
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int u = u0 + ty * 2 + i, v = v0 + tx * 2 + j;
      if (u < n && v < n) o[(long long)u * n + v] = c[i][j];
    }
}

// S[i][j] = dV * (conj(a_i) . b_j) from the real Gram G (n = 2*nst)
__global__ void gram_finalize(const double *partial, int splits, int nst, double dv, double *S) {
  const int i = blockIdx.y, j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nst) return;
  const int n = 2 * nst;
  Kahan re = {0, 0}, im = {0, 0};
  for (int z = 0; z < splits; ++z) {
    const double *G = partial + (long long)z * n * n;
    const double rr = G[(2 * i) * n + 2 * j], ii = G[(2 * i + 1) * n + 2 * j + 1];
    const double ri = G[(2 * i) * n + 2 * j + 1], ir = G[(2 * i + 1) * n + 2 * j];
    kadd(re, rr);
    kadd(re, ii);
    kadd(im, ri);
    kadd(im, -ir);
  }
  S[2 * ((long long)i * nst + j)] = (re.s + re.c) * dv;
  S[2 * ((long long)i * nst + j) + 1] = (im.s + im.c) * dv;
}

// Cholesky S = U^H U (upper) and the inverse of U, one CTA.  S, U, Uinv are
// complex nst x nst row-major (interleaved).  err[0] = 1 if S is not
// positive definite.
__global__ void cholesky_inverse_kernel(const double *S, int nst, double *U, double *Uinv, int *err) {
  const int t = threadIdx.x;
  for (int i = t; i < nst * nst; i += blockDim.x) {
    U[2 * i] = U[2 * i + 1] = 0.0;
    Uinv[2 * i] = Uinv[2 * i + 1] = 0.0;
  }
  __syncthreads();
  __shared__ double djj;
  for (int j = 0; j < nst; ++j) {
    if (t == 0) {
      double d = S[2 * (j * nst + j)];
      for (int k = 0; k < j; ++k) {
        const double ur = U[2 * (k * nst + j)], ui = U[2 * (k * nst + j) + 1];
        d -= ur * ur + ui * ui;
      }
      if (!(d > 0.0)) {
        err[0] = 1;
        d = 1.0;
      }
      djj = sqrt(d);
      U[2 * (j * nst + j)] = djj;
    }
    __syncthreads();
    for (int i = j + 1 + t; i < nst; i += blockDim.x) {
      double sr = S[2 * (j * nst + i)], si = S[2 * (j * nst + i) + 1];
      for (int k = 0; k < j; ++k) {
        const double ar = U[2 * (k * nst + j)], ai = -U[2 * (k * nst + j) + 1];  // conj
        const double br = U[2 * (k * nst + i)], bi = U[2 * (k * nst + i) + 1];
        sr -= ar * br - ai * bi;
        si -= ar * bi + ai * br;
      }
      U[2 * (j * nst + i)] = sr / djj;
      U[2 * (j * nst + i) + 1] = si / djj;
    }
    __syncthreads();
  }
  // Uinv: solve U X = I column by column (thread per column)
  for (int c = t; c < nst; c += blockDim.x) {
    for (int i = c; i >= 0; --i) {
      double xr = (i == c) ? 1.0 : 0.0, xi = 0.0;
      for (int k = i + 1; k <= c; ++k) {
        const double ur = U[2 * (i * nst + k)], ui = U[2 * (i * nst + k) + 1];
        const double vr = Uinv[2 * (k * nst + c)], vi = Uinv[2 * (k * nst + c) + 1];
        xr -= ur * vr - ui * vi;
        xi -= ur * vi + ui * vr;
      }
      const double d = U[2 * (i * nst + i)];
      Uinv[2 * (i * nst + c)] = xr / d;
      Uinv[2 * (i * nst + c) + 1] = xi / d;
    }
  }
}

// psi[p][j] <- sum_{i<=j} psi[p][i] Uinv[i][j]; one CTA per row block.
template <typename T>
__global__ void __launch_bounds__(256) trsm_apply_kernel(T *psi, long long ld, int np, int nst,
                                                        const double *Uinv) {
  using V = typename C2<T>::type;
  extern __shared__ double rowbuf[];  // rows_per_iter x nst complex
  const int t = threadIdx.x;
  const int R = max(1, 256 / nst);  // rows per iteration
  const long long per = (np + gridDim.x - 1) / gridDim.x;
  const long long p0 = blockIdx.x * per, p1 = min((long long)np, p0 + per);
  for (long long pb = p0; pb < p1; pb += R) {
    __syncthreads();
    for (int i = t; i < R * nst; i += blockDim.x) {
      const long long row = pb + i / nst;
      const int s = i % nst;
      if (row < p1) {
        const V x = reinterpret_cast<const V *>(psi + row * 2 * ld)[s];
        rowbuf[2 * i] = double(x.x);
        rowbuf[2 * i + 1] = double(x.y);
      }
    }
    __syncthreads();
    for (int i = t; i < R * nst; i += blockDim.x) {
      const int rr = i / nst, j = i % nst;
      const long long row = pb + rr;
      if (row >= p1) continue;
      double yr = 0.0, yi = 0.0;
      const double *x = rowbuf + 2 * rr * nst;
      for (int k = 0; k <= j; ++k) {
        const double ur = __ldg(Uinv + 2 * (k * nst + j)), ui = __ldg(Uinv + 2 * (k * nst + j) + 1);
        yr = fma(x[2 * k], ur, fma(-x[2 * k + 1], ui, yr));
        yi = fma(x[2 * k], ui, fma(x[2 * k + 1], ur, yi));
      }
      V y;
      y.x = static_cast<decltype(y.x)>(yr);
      y.y = static_cast<decltype(y.y)>(yi);
      reinterpret_cast<V *>(psi + row * 2 * ld)[j] = y;
    }
  }
}

// observables: partial [ncta][ld][3][2] -> out[3][nst] (energy, norm2, dipole) * dv.
// One CTA per state: its threads take strided slices of the CTA partials
// (compensated sums), then fold them in shared memory.
__global__ void __launch_bounds__(128) obs_finalize_kernel(const double *partial, int ncta, int ld, int nst,
                                                           double dv, const double *ket_partial, int nket,
                                                           double *out) {
  const int s = blockIdx.x;
  __shared__ double red[3][2][128];
  Kahan a[3] = {{0, 0}, {0, 0}, {0, 0}};
  for (int c = threadIdx.x; c < ncta; c += blockDim.x) {
    const double *p = partial + ((long long)c * ld + s) * 6;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      kadd(a[q], p[2 * q]);
      a[q].c += p[2 * q + 1];
    }
  }
  if (ket_partial)
    for (int c = threadIdx.x; c < nket; c += blockDim.x) {
      const double *p = ket_partial + ((long long)c * ld + s) * 2;
      kadd(a[0], p[0]);
      a[0].c += p[1];
    }
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    red[q][0][threadIdx.x] = a[q].s;
    red[q][1][threadIdx.x] = a[q].c;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    const int q = threadIdx.x;
    Kahan t = {0, 0};
    for (int i = 0; i < int(blockDim.x); ++i) {
      kadd(t, red[q][0][i]);
      t.c += red[q][1][i];
    }
    out[q * nst + s] = (t.s + t.c) * dv;
  }
}

// rho[ip] (+)= sum_s w[s] |psi_s(ip)|^2 over the np inner points: one warp per
// row, lanes over the states, FP64 sums folded in a fixed order (deterministic).
template <typename T>
__global__ void __launch_bounds__(256) density_kernel(const T *psi, long long ld, int np, int nst, const double *w,
                                                      double *rho, int accumulate) {
  const int lane = threadIdx.x & 31;
  for (long long row = blockIdx.x * 8LL + (threadIdx.x >> 5); row < np; row += gridDim.x * 8LL) {
    const T *r = psi + row * 2 * ld;
    double acc = 0.0;
    for (int s = lane; s < nst; s += 32) {
      const double re = double(r[2 * s]), im = double(r[2 * s + 1]);
      acc += __ldg(w + s) * (re * re + im * im);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (lane == 0) rho[row] = accumulate ? rho[row] + acc : acc;
  }
}

}  // namespace

template <typename T>
hpsi_status launch_density(const T *psi, long long ld, int np, int nst, const double *w, double *rho, int accumulate,
                           cudaStream_t st) {
  if (np < 1) return HPSI_OK;
  const int grid = std::min((np + 7) / 8, 148 * 16);
  density_kernel<T><<<grid, 256, 0, st>>>(psi, ld, np, nst, w, rho, accumulate);
  HPSI_CHECK_LAUNCH();
  return HPSI_OK;
}
template hpsi_status launch_density<double>(const double *, long long, int, int, const double *, double *, int,
                                            cudaStream_t);
template hpsi_status launch_density<float>(const float *, long long, int, int, const double *, double *, int,
                                           cudaStream_t);

int reduce_blocks(int np) {
  int nb = (np + 4095) / 4096;
  return nb < 1 ? 1 : (nb > 1184 ? 1184 : nb);
}

template <typename T>
hpsi_status launch_state_sum(int mode, const T *a, long long lda, const T *b, long long ldb, int np, int nst,
                             double *partial, int nblk, double scale, int sqrt_first, double *out,
                             cudaStream_t st) {
  dim3 grid(nblk, (nst + 255) / 256);
  if (mode == 0)
    state_sum_kernel<T, 0><<<grid, 256, 0, st>>>(a, lda, b, ldb, np, nst, partial);
  else
    state_sum_kernel<T, 1><<<grid, 256, 0, st>>>(a, lda, b, ldb, np, nst, partial);
  HPSI_CHECK_LAUNCH();
  state_sum_finalize<<<(nst + 127) / 128, 128, 0, st>>>(partial, nblk, nst, scale, sqrt_first, out);
  HPSI_CHECK_LAUNCH();
  return HPSI_OK;
}

int gram_splits(int np) {
  int s = (np + 8191) / 8192;
  return s < 1 ? 1 : (s > 256 ? 256 : s);
}

template <typename T>
hpsi_status launch_gram(const T *a, long long lda, const T *b, long long ldb, int np, int nst, double *partial,
                        int splits, double dv, double *S, cudaStream_t st) {
  const int n = 2 * nst;
  dim3 grid((n + 31) / 32, (n + 31) / 32, splits);
  gram_kernel<T><<<grid, dim3(16, 16), 0, st>>>(a, lda, b, ldb, np, n, partial);
  HPSI_CHECK_LAUNCH();
  gram_finalize<<<dim3((nst + 127) / 128, nst), 128, 0, st>>>(partial, splits, nst, dv, S);
  HPSI_CHECK_LAUNCH();
  return HPSI_OK;
}

hpsi_status launch_cholesky_inverse(const double *S, int nst, double *U, double *Uinv, int *err, cudaStream_t st) {
  cholesky_inverse_kernel<<<1, 256, 0, st>>>(S, nst, U, Uinv, err);
  HPSI_CHECK_LAUNCH();
  return HPSI_OK;
}

template <typename T>
hpsi_status launch_trsm_apply(T *psi, long long ld, int np, int nst, const double *Uinv, cudaStream_t st) {
  const int R = nst >= 256 ? 1 : 256 / nst;
  const size_t smem = size_t(R) * nst * 2 * sizeof(double);
  if (smem > 48 * 1024) {
    set_error("orthonormalisation supports at most 1536 states");
    return HPSI_ERR_UNSUPPORTED;
  }
  int nb = (np + 1023) / 1024;
  nb = nb < 1 ? 1 : (nb > 2368 ? 2368 : nb);
  trsm_apply_kernel<T><<<nb, 256, smem, st>>>(psi, ld, np, nst, Uinv);
  HPSI_CHECK_LAUNCH();
  return HPSI_OK;
}

hpsi_status launch_obs_finalize(const double *partial, int ncta, int ld, int nst, double dv,
                                const double *ket_partial, int nket, double *out, cudaStream_t st) {
  if (nst < 1) return HPSI_OK;
  obs_finalize_kernel<<<nst, 128, 0, st>>>(partial, ncta, ld, nst, dv, ket_partial, nket, out);
  HPSI_CHECK_LAUNCH();
  return HPSI_OK;
}

template hpsi_status launch_state_sum<double>(int, const double *, long long, const double *, long long, int, int,
                                              double *, int, double, int, double *, cudaStream_t);
template hpsi_status launch_state_sum<float>(int, const float *, long long, const float *, long long, int, int,
                                             double *, int, double, int, double *, cudaStream_t);
template hpsi_status launch_gram<double>(const double *, long long, const double *, long long, int, int, double *,
                                         int, double, double *, cudaStream_t);
template hpsi_status launch_gram<float>(const float *, long long, const float *, long long, int, int, double *,
                                        int, double, double *, cudaStream_t);
template hpsi_status launch_trsm_apply<double>(double *, long long, int, int, const double *, cudaStream_t);
template hpsi_status launch_trsm_apply<float>(float *, long long, int, int, const double *, cudaStream_t);

}  // namespace hpsi
