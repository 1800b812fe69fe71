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

// RPW mesh rows per warp (32 / RPW lanes per row: 2 or 4 rows for batches of
// at most 16 or 8 states, so lanes past the batch width do not idle), K the
// Taylor order (a template parameter: the per-element terms stay in registers).
// For each state: s = sum_j conj(L_j) Phi_j with
// Phi_j = sum_{m <= K-1-j} c_{j+m+1} P_m; lambda_new = sum_k conj(c_k) L_k
// written over L_0.  w(r) = sum_i Re s_i; gv[r] += 2 dV w; the eps gradient
// partial of the block += 2 dV z(r) w, and the same for the leading term.
template <int K, int RPW>
__global__ void __launch_bounds__(256) adj_accumulate_kernel(double2 *L0, const AdjPtrs ptr, long long ld, int nst,
                                                             int np, const AdjCoef c, const double *zrow, double dv,
                                                             double *gv, double *geps_partial,
                                                             double *gcont_partial) {
  constexpr int LN = 32 / RPW;  // lanes per row
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int sub = lane / LN, li = lane % LN;
  const int rows_per_block = (blockDim.x >> 5) * RPW;
  Kahan ke = {0, 0}, kc = {0, 0};
  for (long long r0 = (long long)blockIdx.x * rows_per_block + warp * RPW; r0 < np;
       r0 += (long long)gridDim.x * rows_per_block) {
    const long long r = r0 + sub;
    const bool rv = r < np;
    double wr = 0.0, wc = 0.0;
    for (int i = li; rv && i < nst; i += LN) {
      const long long o = r * ld + i;
      double2 Pm[K], Lk[K + 1];
#pragma unroll
      for (int m = 0; m < K; ++m) Pm[m] = ptr.P[m][o];
#pragma unroll
      for (int k = 0; k <= K; ++k) Lk[k] = ptr.L[k][o];
      double sre = 0.0;
#pragma unroll
      for (int j = 0; j < K; ++j) {
        double pre = 0.0, pim = 0.0;  // Phi_j
#pragma unroll
        for (int m = 0; m + j <= K - 1; ++m) {
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
#pragma unroll
      for (int k = 0; k <= K; ++k) {
        const double ar = c.cre[k], ai = -c.cim[k];
        nre += ar * Lk[k].x - ai * Lk[k].y;
        nim += ar * Lk[k].y + ai * Lk[k].x;
      }
      L0[o] = make_double2(nre, nim);
    }
    // sum over the row's lanes (xor offsets below LN stay inside the group)
    for (int off = LN / 2; off > 0; off >>= 1) {
      wr += __shfl_xor_sync(0xffffffffu, wr, off);
      wc += __shfl_xor_sync(0xffffffffu, wc, off);
    }
    if (li == 0 && rv) {
      if (gv) gv[r] += 2.0 * dv * wr;
      kadd(ke, 2.0 * dv * wr * zrow[r]);
      kadd(kc, 2.0 * dv * wc * zrow[r]);
    }
  }
  // the row groups' partials into lane 0, in a fixed order
#pragma unroll
  for (int q = 1; q < RPW; ++q) {
    const double es = __shfl_sync(0xffffffffu, ke.s, q * LN), ec = __shfl_sync(0xffffffffu, ke.c, q * LN);
    const double cs = __shfl_sync(0xffffffffu, kc.s, q * LN), cc = __shfl_sync(0xffffffffu, kc.c, q * LN);
    if (lane == 0) {
      kadd(ke, es);
      ke.c += ec;
      kadd(kc, cs);
      kc.c += cc;
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
    for (int w = 0; w < int(blockDim.x >> 5); ++w) {
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

template <int K>
void launch_adj_accumulate(int rpw, unsigned grid, cudaStream_t st, double2 *L0, const AdjPtrs &ptr, long long ld,
                           int nst, int np, const AdjCoef &c, const double *zrow, double dv, double *gv, double *gp,
                           double *gcp) {
  if (rpw == 4)
    adj_accumulate_kernel<K, 4><<<grid, 256, 0, st>>>(L0, ptr, ld, nst, np, c, zrow, dv, gv, gp, gcp);
  else if (rpw == 2)
    adj_accumulate_kernel<K, 2><<<grid, 256, 0, st>>>(L0, ptr, ld, nst, np, c, zrow, dv, gv, gp, gcp);
  else
    adj_accumulate_kernel<K, 1><<<grid, 256, 0, st>>>(L0, ptr, ld, nst, np, c, zrow, dv, gv, gp, gcp);
}

// The two block-partial sums of a step (warp 0: the eps gradient, warp 1: its
// leading-term form): each lane a compensated sum over a stride of the
// partials, then lane 0 over the 32 lane sums in lane order (fixed order:
// deterministic).
__global__ void adj_sum_partials(const double *part, const double *partc, int n, double *out, double *outc) {
  const int lane = threadIdx.x & 31;
  const double *p = threadIdx.x < 32 ? part : partc;
  Kahan a = {0, 0};
  for (int i = lane; i < n; i += 32) {
    kadd(a, p[2 * i]);
    a.c += p[2 * i + 1];
  }
  Kahan t = {0, 0};
  for (int q = 0; q < 32; ++q) {
    const double s = __shfl_sync(0xffffffffu, a.s, q), c = __shfl_sync(0xffffffffu, a.c, q);
    kadd(t, s);
    t.c += c;
  }
  if (lane == 0) *(threadIdx.x < 32 ? out : outc) = t.s + t.c;
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

// pol . r of every inner row (cell coordinates of the padded box)
__global__ void zrow_kernel(const int *cell_of_row, int np, int NX, int NY, int lo0, int lo1, int lo2, double h0,
                            double h1, double h2, double p0, double p1, double p2, double *z) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= np) return;
  const int c = cell_of_row[r];
  const int x = c % NX, y = (c / NX) % NY, zz = c / (NX * NY);
  z[r] = p0 * (x + lo0) * h0 + p1 * (y + lo1) * h1 + p2 * (zz + lo2) * h2;
}

// Per-state partial sums of conj(chi_i(r)) z(r) psi_i(r) over the rows a
// block visits: blockDim = (tx states, ty rows); compensated per thread, the
// ty row groups folded in a fixed order.  partial[block][state] = {re s, re c,
// im s, im c}.
template <typename T>
__global__ void vjp_field_kernel(const T *chi, long long ldc, const T *psi, long long ldp, const double *z, int np,
                                 int nst, double *partial) {
  extern __shared__ double red[];  // ty * tx * 4
  const int tx = blockDim.x, ty = blockDim.y;
  for (int s0 = 0; s0 < nst; s0 += tx) {
    const int s = s0 + threadIdx.x;
    Kahan re = {0, 0}, im = {0, 0};
    if (s < nst)
      for (long long r = (long long)blockIdx.x * ty + threadIdx.y; r < np; r += (long long)gridDim.x * ty) {
        const double cr = chi[2 * (r * ldc + s)], ci = chi[2 * (r * ldc + s) + 1];
        const double pr = psi[2 * (r * ldp + s)], pi = psi[2 * (r * ldp + s) + 1];
        const double zr = z[r];
        kadd(re, zr * (cr * pr + ci * pi));
        kadd(im, zr * (cr * pi - ci * pr));
      }
    double *o = red + 4 * (threadIdx.y * tx + threadIdx.x);
    o[0] = re.s;
    o[1] = re.c;
    o[2] = im.s;
    o[3] = im.c;
    __syncthreads();
    if (threadIdx.y == 0 && s < nst) {
      Kahan a = {0, 0}, b = {0, 0};
      for (int y = 0; y < ty; ++y) {
        const double *q = red + 4 * (y * tx + threadIdx.x);
        kadd(a, q[0]);
        a.c += q[1];
        kadd(b, q[2]);
        b.c += q[3];
      }
      double *d = partial + 4 * ((long long)blockIdx.x * nst + s);
      d[0] = a.s;
      d[1] = a.c;
      d[2] = b.s;
      d[3] = b.c;
    }
    __syncthreads();
  }
}

// out[2 i] + i out[2 i + 1] = scale * sum over the blocks' partials of state i
__global__ void vjp_field_finalize(const double *partial, int nblk, int nst, double scale, double *out) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nst) return;
  Kahan a = {0, 0}, b = {0, 0};
  for (int k = 0; k < nblk; ++k) {
    const double *q = partial + 4 * ((long long)k * nst + s);
    kadd(a, q[0]);
    a.c += q[1];
    kadd(b, q[2]);
    b.c += q[3];
  }
  out[2 * s] = scale * (a.s + a.c);
  out[2 * s + 1] = scale * (b.s + b.c);
}

// g[r] = (acc ? g[r] : 0) + scale * sum_i Re(conj(lam_i(r)) psi_i(r)): one warp
// per row, states over the lanes, a fixed shuffle order
template <typename T>
__global__ void vjp_vloc_kernel(const T *lam, long long ldl, const T *psi, long long ldp, int np, int nst,
                                double scale, int acc, double *g) {
  const int lane = threadIdx.x & 31;
  const long long r = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (r >= np) return;
  double w = 0.0;
  for (int s = lane; s < nst; s += 32) {
    const double lr = lam[2 * (r * ldl + s)], li = lam[2 * (r * ldl + s) + 1];
    const double pr = psi[2 * (r * ldp + s)], pi = psi[2 * (r * ldp + s) + 1];
    w += lr * pr + li * pi;
  }
  for (int off = 16; off > 0; off >>= 1) w += __shfl_xor_sync(0xffffffffu, w, off);
  if (lane == 0) g[r] = (acc ? g[r] : 0.0) + scale * w;
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

// Scratch of one backward step: H^k lambda (k = 1..K), H^m psi (m = 1..K-1),
// z per row and the block partials.
struct AdjStepBufs {
  double2 *L[KMAX + 1];
  double2 *P[KMAX];
  double *zrow, *part, *partc;
};
constexpr int ADJ_NBLK = 296;

static size_t adj_step_bytes(const hpsi_mesh *m, long long ld, int K) {
  const size_t batch = size_t(m->np) * ld;
  return batch * size_t(2 * K - 1) * sizeof(double2) + (size_t(m->np) + 4 * ADJ_NBLK + 8) * sizeof(double);
}

static AdjStepBufs adj_step_carve(void *base, const hpsi_mesh *m, long long ld, int K) {
  AdjStepBufs B;
  std::memset(&B, 0, sizeof(B));
  const size_t batch = size_t(m->np) * ld;
  double2 *q = static_cast<double2 *>(base);
  for (int k = 1; k <= K; ++k, q += batch) B.L[k] = q;
  for (int k = 1; k < K; ++k, q += batch) B.P[k] = q;
  B.zrow = reinterpret_cast<double *>(q);
  B.part = B.zrow + m->np;
  B.partc = B.part + 2 * ADJ_NBLK;
  return B;
}

static hpsi_status adj_zrow(const hpsi_mesh *m, const double pol[3], double *z, cudaStream_t st) {
  const CellBox &b = m->box;
  zrow_kernel<<<(m->np + 255) / 256, 256, 0, st>>>(m->d_cell_of_row, m->np, b.NX, b.NY, b.lo[0], b.lo[1], b.lo[2],
                                                  b.h[0], b.h[1], b.h[2], pol[0], pol[1], pol[2], z);
  HPSI_CHECK_LAUNCH();
  return HPSI_OK;
}

// One backward step of the exact discrete adjoint: lam <- T_n^dagger lam in
// place (lam = lambda_{n+1} on entry), with psi = psi_n the state the forward
// step n started from; adds the step's dJ/d eps_n into geps[0] and the
// leading (continuous-adjoint) term into gcont[0] (device scalars, written),
// and dJ/dv(r) into gv (device, accumulated; may be null).  B.zrow holds
// pol . r.
static hpsi_status adjoint_step_dev(const AdjointRun &R, double eps, double2 *lam, const double2 *psi,
                                    const AdjStepBufs &B, double *geps, double *gcont, double *gv) {
  AdjCoef coef;
  coef.K = R.K;
  std::complex<double> ck(1.0, 0.0);
  for (int k = 0; k <= R.K; ++k) {
    if (k > 0) ck *= std::complex<double>(0.0, -R.dt) / double(k);
    coef.cre[k] = ck.real();
    coef.cim[k] = ck.imag();
  }
  AdjPtrs ptr;
  std::memset(&ptr, 0, sizeof(ptr));
  ptr.L[0] = lam;
  ptr.P[0] = psi;
  for (int k = 1; k <= R.K; ++k) ptr.L[k] = B.L[k];
  for (int k = 1; k < R.K; ++k) ptr.P[k] = B.P[k];
  hpsi_status s = HPSI_OK;
  for (int k = 1; k < R.K && !s; ++k) s = adj_apply(R, eps, ptr.P[k - 1], B.P[k]);
  for (int k = 1; k <= R.K && !s; ++k) s = adj_apply(R, eps, ptr.L[k - 1], B.L[k]);
  if (s) return s;
  const double dv = R.h->mesh->box.h[0] * R.h->mesh->box.h[1] * R.h->mesh->box.h[2];
  const int rpw = R.nst <= 8 ? 4 : R.nst <= 16 ? 2 : 1;
  switch (R.K) {
#define HPSI_ADJ_ACC(KK)                                                                                      \
  case KK:                                                                                                    \
    launch_adj_accumulate<KK>(rpw, ADJ_NBLK, R.st, lam, ptr, R.ld, R.nst, R.np, coef, B.zrow, dv, gv, B.part, \
                              B.partc);                                                                       \
    break;
    HPSI_ADJ_ACC(1)
    HPSI_ADJ_ACC(2)
    HPSI_ADJ_ACC(3)
    HPSI_ADJ_ACC(4)
    HPSI_ADJ_ACC(5)
    HPSI_ADJ_ACC(6)
    HPSI_ADJ_ACC(7)
    HPSI_ADJ_ACC(8)
#undef HPSI_ADJ_ACC
    default:
      set_error("adjoint step: Taylor order out of range");
      return HPSI_ERR_ARG;
  }
  HPSI_CHECK_LAUNCH();
  adj_sum_partials<<<1, 64, 0, R.st>>>(B.part, B.partc, ADJ_NBLK, geps, gcont);
  HPSI_CHECK_LAUNCH();
  return HPSI_OK;
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
  // complex buffers: checkpoints nseg, segment seglen, lambda; then the step
  // scratch; doubles: gv np, ov 2*ld, ov partial 4*ld, geps nsteps, gcont nsteps
  const size_t ncplx = batch * (size_t(nseg) + seglen + 1);
  const size_t ndbl = size_t(m->np) + 6 * size_t(R.ld) + 2 * size_t(nsteps) + 8;
  const size_t stepb = adj_step_bytes(m, R.ld, order);
  hpsi_status s = h->adjbuf.ensure(ncplx * sizeof(double2) + ndbl * sizeof(double) + 256 + stepb);
  if (s) return s;
  double2 *ckp = static_cast<double2 *>(h->adjbuf.ptr);
  double2 *seg = ckp + batch * nseg;
  double2 *Lb = seg + batch * seglen;
  double *gv = reinterpret_cast<double *>(Lb + batch);
  double *ov = gv + m->np;           // 2*ld
  double *ovpart = ov + 2 * R.ld;    // 4*ld (state_sum partial of one block)
  double *geps = ovpart + 4 * R.ld;  // nsteps
  double *gcont = geps + nsteps;     // nsteps
  // the step scratch starts on the next 256-byte boundary (room reserved above)
  void *stepbase = reinterpret_cast<void *>((reinterpret_cast<uintptr_t>(gcont + nsteps + 8) + 255) &
                                            ~uintptr_t(255));
  const AdjStepBufs B = adj_step_carve(stepbase, m, R.ld, order);
  s = adj_zrow(m, pol, B.zrow, st);
  if (s) return s;
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
      s = adjoint_step_dev(R, eps[n], Lb, seg + batch * (n - n0), B, geps + n, gcont + n, gv);
      if (s) return fail(s);
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

// ---------------------------------------------------------------------------
// Per-step primitives for a host-driven backward propagation (bwd_step /
// bwd_step_2, src/opt_control/propagation.F90:477-783).

static hpsi_status adj_check_pair(const hpsi_mesh *m, const hpsi_batch *a, const hpsi_batch *b, bool c128_only,
                                  const char *who) {
  if (!a || !b || !a->ptr || !b->ptr || a->dtype != b->dtype || a->nst != b->nst || a->nst < 1 ||
      a->ld < a->nst || b->ld < b->nst || a->npts < m->np || b->npts < m->np || !is_device_ptr(a->ptr) ||
      !is_device_ptr(b->ptr) || (a->dtype != HPSI_C128 && a->dtype != HPSI_C64) ||
      (c128_only && a->dtype != HPSI_C128)) {
    set_error(std::string(who) + ": two device batches of one dtype" + (c128_only ? " (complex128)" : "") +
              ", equal nst and at least np rows expected");
    return HPSI_ERR_ARG;
  }
  return HPSI_OK;
}

extern "C" hpsi_status hpsi_adjoint_step(hpsi_hamiltonian *h, hpsi_batch *lambda, const hpsi_batch *psi_n,
                                         double eps_n, const double pol[3], double dt, int32_t order,
                                         double *grad_eps, double *grad_eps_cont, double *grad_v, void *stream) {
  if (!h || !pol || !(dt > 0.0) || order < 1 || order > KMAX || !std::isfinite(eps_n)) {
    set_error("hpsi_adjoint_step: bad argument");
    return HPSI_ERR_ARG;
  }
  hpsi_mesh *m = h->mesh;
  hpsi_status s = adj_check_pair(m, lambda, psi_n, true, "hpsi_adjoint_step");
  if (s) return s;
  if (lambda->ld != psi_n->ld) {
    set_error("hpsi_adjoint_step: lambda and psi_n must have the same ld");
    return HPSI_ERR_ARG;
  }
  if (!h->have_kinetic) {
    set_error("hpsi_adjoint_step: kinetic weights not set");
    return HPSI_ERR_STATE;
  }
  if (grad_v && !is_device_ptr(grad_v)) {
    set_error("hpsi_adjoint_step: grad_v must be device memory (np doubles, accumulated)");
    return HPSI_ERR_ARG;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  AdjointRun R{h, lambda->ld, lambda->nst, m->np, order, dt, {pol[0], pol[1], pol[2]}, st};
  const size_t stepb = adj_step_bytes(m, R.ld, order);
  s = h->adjstep.ensure(stepb + 4 * sizeof(double));
  if (s) return s;
  const AdjStepBufs B = adj_step_carve(h->adjstep.ptr, m, R.ld, order);
  double *g2 = reinterpret_cast<double *>(static_cast<char *>(h->adjstep.ptr) + stepb);
  s = adj_zrow(m, pol, B.zrow, st);
  if (s) return s;
  const double save_fld[3] = {h->fld[0], h->fld[1], h->fld[2]};
  s = adjoint_step_dev(R, eps_n, static_cast<double2 *>(lambda->ptr), static_cast<const double2 *>(psi_n->ptr), B,
                       g2, g2 + 1, grad_v);
  for (int a = 0; a < 3; ++a) h->fld[a] = save_fld[a];
  if (s) return s;
  bool host_out = false;
  for (double *o : {grad_eps, grad_eps_cont})
    if (o) {
      HPSI_TRY_CUDA(cudaMemcpyAsync(o, o == grad_eps ? g2 : g2 + 1, sizeof(double), cudaMemcpyDefault, st));
      host_out = host_out || !is_device_ptr(o);
    }
  if (host_out) HPSI_TRY_CUDA(cudaStreamSynchronize(st));
  return HPSI_OK;
}

extern "C" hpsi_status hpsi_vjp_field(hpsi_hamiltonian *h, const hpsi_batch *chi, const hpsi_batch *psi,
                                      const double pol[3], double *out, void *stream) {
  if (!h || !pol || !out) {
    set_error("hpsi_vjp_field: bad argument");
    return HPSI_ERR_ARG;
  }
  hpsi_mesh *m = h->mesh;
  hpsi_status s = adj_check_pair(m, chi, psi, false, "hpsi_vjp_field");
  if (s) return s;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int nst = chi->nst;
  const int tx = nst >= 32 ? 32 : nst, ty = 256 / tx;
  const int nblk = std::max(1, std::min(2 * m->num_sms, (m->np + ty - 1) / ty));
  const size_t part_d = size_t(nblk) * nst * 4, out_d = 2 * size_t(nst);
  s = h->vjpbuf.ensure((size_t(m->np) + part_d + out_d) * sizeof(double));
  if (s) return s;
  double *z = static_cast<double *>(h->vjpbuf.ptr), *part = z + m->np, *res = part + part_d;
  s = adj_zrow(m, pol, z, st);
  if (s) return s;
  const size_t shm = size_t(tx) * ty * 4 * sizeof(double);
  if (chi->dtype == HPSI_C128)
    vjp_field_kernel<double><<<nblk, dim3(tx, ty), shm, st>>>(static_cast<const double *>(chi->ptr), chi->ld,
                                                             static_cast<const double *>(psi->ptr), psi->ld, z,
                                                             m->np, nst, part);
  else
    vjp_field_kernel<float><<<nblk, dim3(tx, ty), shm, st>>>(static_cast<const float *>(chi->ptr), chi->ld,
                                                            static_cast<const float *>(psi->ptr), psi->ld, z, m->np,
                                                            nst, part);
  HPSI_CHECK_LAUNCH();
  const double dv = m->box.h[0] * m->box.h[1] * m->box.h[2];
  vjp_field_finalize<<<(nst + 127) / 128, 128, 0, st>>>(part, nblk, nst, dv, res);
  HPSI_CHECK_LAUNCH();
  HPSI_TRY_CUDA(cudaMemcpyAsync(out, res, out_d * sizeof(double), cudaMemcpyDefault, st));
  if (!is_device_ptr(out)) HPSI_TRY_CUDA(cudaStreamSynchronize(st));
  return HPSI_OK;
}

extern "C" hpsi_status hpsi_vjp_vloc(hpsi_hamiltonian *h, const hpsi_batch *lambda, const hpsi_batch *psi,
                                     double scale, double *grad_v, int32_t accumulate, void *stream) {
  if (!h || !grad_v || !std::isfinite(scale)) {
    set_error("hpsi_vjp_vloc: bad argument");
    return HPSI_ERR_ARG;
  }
  hpsi_mesh *m = h->mesh;
  hpsi_status s = adj_check_pair(m, lambda, psi, false, "hpsi_vjp_vloc");
  if (s) return s;
  if (!is_device_ptr(grad_v)) {
    set_error("hpsi_vjp_vloc: grad_v must be device memory (np doubles)");
    return HPSI_ERR_ARG;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const unsigned nb = unsigned((m->np + 7) / 8);
  if (lambda->dtype == HPSI_C128)
    vjp_vloc_kernel<double><<<nb, 256, 0, st>>>(static_cast<const double *>(lambda->ptr), lambda->ld,
                                                static_cast<const double *>(psi->ptr), psi->ld, m->np, lambda->nst,
                                                scale, accumulate ? 1 : 0, grad_v);
  else
    vjp_vloc_kernel<float><<<nb, 256, 0, st>>>(static_cast<const float *>(lambda->ptr), lambda->ld,
                                               static_cast<const float *>(psi->ptr), psi->ld, m->np, lambda->nst,
                                               scale, accumulate ? 1 : 0, grad_v);
  HPSI_CHECK_LAUNCH();
  return HPSI_OK;
}
