/*
 * CPU ORACLE -- test infrastructure only.
 *
 * This file is a plain-C/OpenMP restatement of the reference (Octopus 13.0)
 * FP64 CPU path for the Hamiltonian apply and the Taylor exponential.  It is
 * the checker for the CUDA library and the timed CPU baseline; nothing in the
 * product links it.  Only tests, the smoke check and the benchmark's CPU legs
 * load it.
 *
 * Restated functions (reference file:line):
 *   orc_nl_operator_build  src/grid/nl_operator.F90:308-456 (run compression of
 *                          the stencil offsets, compact boundaries off)
 *   orc_operate_ri         src/grid/operate_inc.c:29-342 (const weights,
 *                          packed batch, runs [imin, imax))
 *   orc_boundaries_set     src/grid/boundaries_inc.F90:331-360 (zero) and
 *                          :650-700 (periodic copy x phase correction)
 *   orc_hpsi               src/hamiltonian/hamiltonian_elec_inc.F90:77-261
 *                          (kinetic -1/2 * Laplacian, vpsi
 *                          hamiltonian_elec_base_inc.F90:233-242, KB projector
 *                          bra :650-780 and ket :909-1027)
 *   orc_taylor             src/electrons/exponential.F90:677-757
 *
 * When the reference's own stencil kernel has been compiled into
 * oracle/_ref (see oracle/Makefile) the caller may pass it as the operate
 * function; otherwise orc_operate_ri is used.
 */
#include <complex.h>
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef void (*operate_fn)(const int *opn, const double *w, const int *opnri,
                           const int *opri, const int *rimap_inv,
                           const int *rimap_inv_max, const double *fi,
                           const int *ldfp, double *fo);

/* ------------------------------------------------------------------ */
/* nl_operator_build: compress per-point offsets into runs.
 * nbr[ii*W + j] is the 0-based mesh index of point ii + stencil point j.
 * Offsets are stored relative to the point, as in op%ri.  Pass ri == NULL to
 * only count.  Returns nri. */
int orc_nl_operator_build(int np, int W, const int *nbr, int *ri, int *rimap,
                          int *rimap_inv) {
  int *st1 = (int *)calloc((size_t)W, sizeof(int));
  int *st2 = (int *)calloc((size_t)W, sizeof(int));
  int nri = 0;
  int current = -1;
  for (int ii = 0; ii < np; ii++) {
    int change = 0, touches = 0, prev_clear = 1;
    for (int j = 0; j < W; j++) {
      st1[j] = nbr[(size_t)ii * W + j] - ii;
      if (st1[j] != st2[j]) change = 1;
      if (ii + st1[j] >= np) touches = 1;
      if (ii - 1 + st2[j] >= np) prev_clear = 0;
    }
    int force_change = touches && prev_clear;
    if (change || force_change) {
      memcpy(st2, st1, sizeof(int) * (size_t)W);
      current++;
      if (ri) memcpy(ri + (size_t)current * W, st1, sizeof(int) * (size_t)W);
    }
    if (rimap) rimap[ii] = current;
  }
  nri = current + 1;
  if (rimap && rimap_inv) {
    rimap_inv[0] = 0;
    for (int ii = 0; ii < np; ii++) rimap_inv[rimap[ii] + 1] = ii + 1;
    rimap_inv[nri] = np;
  }
  free(st1);
  free(st2);
  return nri;
}

/* ------------------------------------------------------------------ */
/* Plain restatement of doperate_ri_vec: fo[(i<<ldf)+k] =
 * sum_j w[j] * fi[((i + ri[l*n+j]) << ldf) + k], j summed in order. */
void orc_operate_ri(const int *opn, const double *w, const int *opnri,
                    const int *opri, const int *rimap_inv,
                    const int *rimap_inv_max, const double *fi,
                    const int *ldfp, double *fo) {
  const ptrdiff_t n = opn[0], nri = opnri[0], ldf = ldfp[0];
  const ptrdiff_t width = (ptrdiff_t)1 << ldf;
  for (ptrdiff_t l = 0; l < nri; l++) {
    const int *index = opri + n * l;
    for (ptrdiff_t i = rimap_inv[l]; i < rimap_inv_max[l]; i++) {
      for (ptrdiff_t k = 0; k < width; k++) {
        double a = 0.0;
        for (ptrdiff_t j = 0; j < n; j++)
          a = fma(w[j], fi[((i + index[j]) << ldf) + k], a);
        fo[(i << ldf) + k] = a;
      }
    }
  }
}

/* ------------------------------------------------------------------ */
typedef struct {
  int np, np_part;
  int ld;    /* packed width in complex numbers (pow2 >= nst) */
  int nst;   /* states actually in use */
  int W;     /* stencil size */
  const double *wre; /* W weights already multiplied by -1/2 */
  int nri;
  const int *ri, *imin, *imax;
  const double *v;   /* np local potential */
  int bc;            /* 0: boundaries as given, 1: zero, 2: periodic */
  const int *per_inner;          /* np_part-np */
  const double *phase_corr;      /* 2*(np_part-np) or NULL */
  /* KB projector matrices (concatenated) */
  int nmat;
  const int *pm_npoints, *pm_nprojs;
  const long long *pm_map_off, *pm_mat_off, *pm_scal_off;
  const int *pm_map;       /* 0-based mesh indices */
  const double *pm_mat;    /* npoints x nprojs, point fastest */
  const double *pm_scal;
  int nthreads;
  operate_fn operate;
} orc_ctx;

static int ilog2(int x) {
  int l = 0;
  while ((1 << l) < x) l++;
  return l;
}

void orc_boundaries_set(const orc_ctx *c, double *psi) {
  const size_t ld2 = 2 * (size_t)c->ld;
  const int nb = c->np_part - c->np;
  if (c->bc == 1) {
    memset(psi + (size_t)c->np * ld2, 0, sizeof(double) * ld2 * (size_t)nb);
  } else if (c->bc == 2) {
#pragma omp parallel for num_threads(c->nthreads) schedule(static)
    for (int b = 0; b < nb; b++) {
      const double *src = psi + (size_t)c->per_inner[b] * ld2;
      double *dst = psi + (size_t)(c->np + b) * ld2;
      if (!c->phase_corr) {
        for (size_t k = 0; k < ld2; k++) dst[k] = src[k];
      } else {
        double pr = c->phase_corr[2 * b], pi = c->phase_corr[2 * b + 1];
        for (int s = 0; s < c->ld; s++) {
          double xr = src[2 * s], xi = src[2 * s + 1];
          dst[2 * s] = xr * pr - xi * pi;
          dst[2 * s + 1] = xr * pi + xi * pr;
        }
      }
    }
  }
}

/* projection[(m_proj_base + iproj) * 2*ld + r] real view, r over 2*ld */
static void orc_bra(const orc_ctx *c, const double *psi, double *proj) {
  const size_t ld2 = 2 * (size_t)c->ld;
#pragma omp parallel for num_threads(c->nthreads) schedule(dynamic)
  for (int m = 0; m < c->nmat; m++) {
    const int npts = c->pm_npoints[m], npr = c->pm_nprojs[m];
    const int *map = c->pm_map + c->pm_map_off[m];
    const double *P = c->pm_mat + c->pm_mat_off[m];
    const double *scal = c->pm_scal + c->pm_scal_off[m];
    double *out = proj + (size_t)c->pm_scal_off[m] * ld2;
    for (int j = 0; j < npr; j++) {
      double *o = out + (size_t)j * ld2;
      for (size_t r = 0; r < ld2; r++) o[r] = 0.0;
      for (int ip = 0; ip < npts; ip++) {
        const double p = P[(size_t)j * npts + ip];
        const double *x = psi + (size_t)map[ip] * ld2;
        for (size_t r = 0; r < ld2; r++) o[r] += x[r] * p;
      }
      for (size_t r = 0; r < ld2; r++) o[r] *= scal[j];
    }
  }
}

static void orc_ket(const orc_ctx *c, const double *proj, double *hpsi) {
  const size_t ld2 = 2 * (size_t)c->ld;
  /* matrices are applied one after the other (the reference loops imat
   * serially and parallelises inside); points of one matrix are distinct. */
  for (int m = 0; m < c->nmat; m++) {
    const int npts = c->pm_npoints[m], npr = c->pm_nprojs[m];
    const int *map = c->pm_map + c->pm_map_off[m];
    const double *P = c->pm_mat + c->pm_mat_off[m];
    const double *in = proj + (size_t)c->pm_scal_off[m] * ld2;
#pragma omp parallel for num_threads(c->nthreads) schedule(static)
    for (int ip = 0; ip < npts; ip++) {
      double *y = hpsi + (size_t)map[ip] * ld2;
      for (size_t r = 0; r < ld2; r++) {
        double a = 0.0;
        for (int j = 0; j < npr; j++) a += in[(size_t)j * ld2 + r] * P[(size_t)j * npts + ip];
        y[r] += a;
      }
    }
  }
}

long long orc_nprojections(const orc_ctx *c) {
  long long n = 0;
  for (int m = 0; m < c->nmat; m++) n += c->pm_nprojs[m];
  return n;
}

/* H psi.  psi: np_part x ld complex (boundary region is written when bc != 0);
 * hpsi: np x ld complex.  proj_scratch: nprojections x ld complex (or NULL). */
void orc_hpsi(const orc_ctx *c, double *psi, double *hpsi, double *proj_scratch) {
  const size_t ld2 = 2 * (size_t)c->ld;
  const int ldf = ilog2(2 * c->ld);
  orc_boundaries_set(c, psi);
  if (c->nmat > 0 && proj_scratch) orc_bra(c, psi, proj_scratch);
  /* kinetic: runs split over threads as multicomm_divide_range_omp does */
  operate_fn op = c->operate ? c->operate : orc_operate_ri;
#pragma omp parallel num_threads(c->nthreads)
  {
    int nth = 1, tid = 0;
#ifdef _OPENMP
    nth = omp_get_num_threads();
    tid = omp_get_thread_num();
#endif
    int ini = (int)(((long long)c->nri * tid) / nth);
    int end = (int)(((long long)c->nri * (tid + 1)) / nth);
    int nloc = end - ini;
    if (nloc > 0)
      op(&c->W, c->wre, &nloc, c->ri + (size_t)ini * c->W, c->imin + ini,
         c->imax + ini, psi, &ldf, hpsi);
  }
  /* local potential */
  if (c->v) {
#pragma omp parallel for num_threads(c->nthreads) schedule(static)
    for (int ip = 0; ip < c->np; ip++) {
      const double vv = c->v[ip];
      const double *x = psi + (size_t)ip * ld2;
      double *y = hpsi + (size_t)ip * ld2;
      for (size_t r = 0; r < ld2; r++) y[r] += vv * x[r];
    }
  }
  if (c->nmat > 0 && proj_scratch) orc_ket(c, proj_scratch, hpsi);
}

/* exponential_taylor_series_batch (no psib2 / inhomogeneous term).
 * deltat is complex (dt_re, dt_im).  psi: np_part x ld (updated in place on
 * the first np points), tmp1/tmp2: np_part x ld scratch. */
void orc_taylor(const orc_ctx *c, double *psi, double dt_re, double dt_im,
                int order, double *psi1, double *hpsi1, double *proj_scratch) {
  const size_t ld2 = 2 * (size_t)c->ld;
  double complex deltat = dt_re + I * dt_im;
  double complex zfact = 1.0;
  int zfact_is_real = fabs(cimag(deltat)) < 2.220446049250313e-16;
  for (int iter = 1; iter <= order; iter++) {
    zfact = zfact * (-I * deltat) / (double)iter;
    zfact_is_real = !zfact_is_real;
    if (iter != 1)
      orc_hpsi(c, psi1, hpsi1, proj_scratch);
    else
      orc_hpsi(c, psi, hpsi1, proj_scratch);
    const double zr = creal(zfact), zi = cimag(zfact);
#pragma omp parallel for num_threads(c->nthreads) schedule(static)
    for (int ip = 0; ip < c->np; ip++) {
      double *y = psi + (size_t)ip * ld2;
      const double *x = hpsi1 + (size_t)ip * ld2;
      if (zfact_is_real) {
        for (size_t r = 0; r < ld2; r++) y[r] += zr * x[r];
      } else {
        for (int s = 0; s < c->ld; s++) {
          double xr = x[2 * s], xi = x[2 * s + 1];
          y[2 * s] += zr * xr - zi * xi;
          y[2 * s + 1] += zr * xi + zi * xr;
        }
      }
    }
    if (iter != order)
      memcpy(psi1, hpsi1, sizeof(double) * ld2 * (size_t)c->np);
  }
}

int orc_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
