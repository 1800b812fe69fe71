// FP64 batch reductions (see reduce.cu).
#pragma once

#include "common.cuh"

namespace hpsi {

int reduce_blocks(int np);
int gram_splits(int np);

// mode 0: out[2*s] = scale * sum |a_s|^2 (sqrt if sqrt_first); mode 1:
// out[2*s], out[2*s+1] = scale * sum conj(a_s) b_s.  partial: nblk*nst*4 doubles.
template <typename T>
hpsi_status launch_state_sum(int mode, const T *a, long long lda, const T *b, long long ldb, int np, int nst,
                             double *partial, int nblk, double scale, int sqrt_first, double *out,
                             cudaStream_t st);

// S (complex nst x nst, interleaved) = dv * a^H b.  partial: splits*(2nst)^2 doubles.
template <typename T>
hpsi_status launch_gram(const T *a, long long lda, const T *b, long long ldb, int np, int nst, double *partial,
                        int splits, double dv, double *S, cudaStream_t st);

hpsi_status launch_cholesky_inverse(const double *S, int nst, double *U, double *Uinv, int *err, cudaStream_t st);

template <typename T>
hpsi_status launch_trsm_apply(T *psi, long long ld, int np, int nst, const double *Uinv, cudaStream_t st);

// partial [ncta][ld][3][2] -> out[3][nst] = (energy, norm2, dipole) * dv;
// ket_partial [nket][ld][2] (may be null) adds the KB part of the energy
// rho[ip] (+)= sum_s w[s] |psi_s(ip)|^2 (w on the device, nst entries)
template <typename T>
hpsi_status launch_density(const T *psi, long long ld, int np, int nst, const double *w, double *rho, int accumulate,
                           cudaStream_t st);

hpsi_status launch_obs_finalize(const double *partial, int ncta, int ld, int nst, double dv,
                                const double *ket_partial, int nket, double *out, cudaStream_t st);

}  // namespace hpsi
