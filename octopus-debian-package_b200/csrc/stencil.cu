// Fused H.psi stencil pass for sm_100a.
//
// One CTA owns a TX x TY column of cells, a block of zb output planes and SC
// complex states (L = 2*SC real lanes).  It marches along z: every plane of
// its column plus a 4-cell halo in x and y is gathered from the packed batch
// into shared memory through a NBUF-deep cp.async ring (rows are found through
// the cell map, so any mesh point order works and each row chunk is one
// contiguous 16..64-byte transfer).  Each thread owns RY consecutive y cells of
// one x column and one real lane, and keeps 9 running sums per cell: when
// plane p arrives it adds w_z(p - z) * psi(p) to the sums of outputs
// z = p-4..p+4 and the x/y arms plus the centre (w_c + v) to output p.  The
// sum of output p-4 is then complete and is written out (for a Taylor pass
// after the Horner update psi0 + a * H u).  The KB ket is added by the
// separate row kernel in projector.cu.
//
// Reference semantics: X(nl_operator_operate_batch)
// (src/grid/nl_operator_inc.F90:21-130) with weights op%w * (-1/2),
// X(hamiltonian_elec_base_local_sub) (src/hamiltonian/hamiltonian_elec_base_inc.F90:233-242),
// the projector ket (:909-1027) and the Taylor axpys
// (src/electrons/exponential.F90:738-746).  Sums are taken in a different
// order than the reference's (rounding differences at the 1e-16 level).
#include <algorithm>
#include <cstdio>
#include <type_traits>

#include "stencil.cuh"

namespace hpsi {

namespace {

template <typename T>
struct Vec16;
template <>
struct Vec16<double> {
  using type = double2;
};
template <>
struct Vec16<float> {
  using type = float4;
};

__device__ __forceinline__ void zero16(void *d) {
  *reinterpret_cast<float4 *>(d) = make_float4(0.f, 0.f, 0.f, 0.f);
}

// copy `bytes` (16, 8 or 4) from global to shared asynchronously
template <int BYTES>
__device__ __forceinline__ void cp_async_n(void *s, const void *g) {
  if constexpr (BYTES == 16)
    cp_async16(s, g);
  else if constexpr (BYTES == 8)
    cp_async8(s, g);
  else
    cp_async4(s, g);
}
template <int BYTES>
__device__ __forceinline__ void zero_n(void *d) {
  if constexpr (BYTES == 16)
    zero16(d);
  else if constexpr (BYTES == 8)
    *reinterpret_cast<float2 *>(d) = make_float2(0.f, 0.f);
  else
    *reinterpret_cast<float *>(d) = 0.f;
}

// complex number of the storage type and its multiply-add by a real weight
template <typename T>
struct Cx;
template <>
struct Cx<double> {
  using type = double2;
};
template <>
struct Cx<float> {
  using type = float2;
};
__device__ __forceinline__ double2 cfma(double w, double2 x, double2 a) {
  return make_double2(fma(w, x.x, a.x), fma(w, x.y, a.y));
}
__device__ __forceinline__ float2 cfma(float w, float2 x, float2 a) {
  return __ffma2_rn(make_float2(w, w), x, a);  // packed FP32 FMA (sm_100)
}
template <typename T>
__device__ __forceinline__ const T *wsel(const double *d, const float *f);
template <>
__device__ __forceinline__ const double *wsel<double>(const double *d, const float *) {
  return d;
}
template <>
__device__ __forceinline__ const float *wsel<float>(const double *, const float *f) {
  return f;
}
template <typename C2>
__device__ __forceinline__ C2 czero() {
  C2 z;
  z.x = 0;
  z.y = 0;
  return z;
}

template <typename T, int SC, int TX, int TY, int RY>
struct PassLayout {
  using C2 = typename Cx<T>::type;
  static constexpr int HAL = 4;
  static constexpr int NBUF = 3;             // data ring; 3 divides the 9-plane unroll
  static constexpr int RING = 9;             // row ring (rows live from load to emission)
  static constexpr int HX = TX + 2 * HAL, HY = TY + 2 * HAL;
  static constexpr int NT = SC * TX * (TY / RY);
  static constexpr int PLANE = HY * HX * SC;  // complex numbers of one halo plane
  static constexpr int INNER = TY * TX * SC;  // complex numbers of one interior plane
  static constexpr size_t off_planes = 0;
  static constexpr size_t off_psi0 = off_planes + size_t(NBUF) * PLANE * sizeof(C2);
  static constexpr size_t off_v = off_psi0 + size_t(NBUF) * INNER * sizeof(C2);
  static constexpr size_t off_rows = off_v + size_t(NBUF) * TY * TX * sizeof(double);
  static constexpr size_t off_maps = off_rows + size_t(RING) * TY * TX * sizeof(int);
  static constexpr size_t bytes = off_maps + size_t(NBUF) * HY * HX * sizeof(int);
};

// Each thread owns one complex state (re and im together) of RY consecutive
// y cells of one x column.  The plane loop is unrolled nine times, so every
// ring position (data, rows, maps, the 9 running sums) is a compile-time
// constant.  HORNER: out = psi0 + a * H in; OBS: per-state observables of in.
template <typename T, int SC, int TX, int TY, int RY, bool HORNER, bool OBS>
__device__ __forceinline__ void pass_body(const PassArgs &p, const int item, const int chunk,
                                          unsigned char *smem) {
  using LY = PassLayout<T, SC, TX, TY, RY>;
  using C2 = typename LY::C2;
  constexpr int HAL = LY::HAL, HX = LY::HX, HY = LY::HY, NT = LY::NT, NBUF = LY::NBUF, RING = LY::RING;
  constexpr int PLANE = LY::PLANE, INNER = LY::INNER;
  constexpr int CELLB = SC * int(sizeof(C2));   // bytes per cell chunk
  constexpr int COPYB = CELLB >= 16 ? 16 : CELLB;
  constexpr int CPC = CELLB / COPYB;            // copies per cell
  constexpr int COPYC = COPYB / int(sizeof(T)); // T elements per copy
  static_assert(NT % CPC == 0, "copy pieces must tile the threads");
  constexpr int CSTEP = NT / CPC;               // cells per copy round
  constexpr int HROUNDS = (HY * HX) / CSTEP, HREM = (HY * HX) % CSTEP;
  constexpr int IROUNDS = (TY * TX) / CSTEP, IREM = (TY * TX) % CSTEP;
  constexpr int NV = TY * TX / 2, NR = TY * TX / 4, NM = HY * HX / 4;  // 16-byte copies
  constexpr bool X0 = HORNER || OBS;

  C2 *planes = reinterpret_cast<C2 *>(smem + LY::off_planes);
  C2 *psi0ring = reinterpret_cast<C2 *>(smem + LY::off_psi0);
  double *vring = reinterpret_cast<double *>(smem + LY::off_v);
  int *rowring = reinterpret_cast<int *>(smem + LY::off_rows);
  int *mapring = reinterpret_cast<int *>(smem + LY::off_maps);

  const int tid = threadIdx.x;
  const int cs = tid % SC;  // complex state within the chunk
  const int tx = (tid / SC) % TX;
  const int tyg = tid / (SC * TX);
  const int4 it = p.items[item];
  const CellBox &B = p.box;
  const int cx0 = HAL + it.x * TX, cy0 = HAL + it.y * TY;
  const int zs = it.z, ze = it.w;
  const long long planeN = (long long)B.NX * B.NY;
  const int zbeg = zs - HAL, zend = ze + HAL;  // planes [zbeg, zend)

  // per-thread copy roles (fixed for the whole kernel)
  const int cell0 = tid / CPC, part = tid % CPC;
  const T *in_base = static_cast<const T *>(p.in) + chunk * SC * 2 + part * COPYC;
  const long long in_ld2 = 2 * p.in_ld;
  const T *psi0_base = static_cast<const T *>(p.psi0) + chunk * SC * 2 + part * COPYC;
  const long long psi0_ld2 = 2 * p.psi0_ld;
  // side copies (16-byte pieces): v (NV), rows (NR), maps (NM); a thread does
  // pieces tid, tid + NT, ... (one round when NT >= NV + NR + NM)
  constexpr int NSIDE = NV + NR + NM;
  constexpr int SROUNDS = (NSIDE + NT - 1) / NT;
  const long long tile0 = (long long)cy0 * B.NX + cx0;
  int side_dst[SROUNDS], side_kind[SROUNDS];
  long long side_src[SROUNDS];
#pragma unroll
  for (int k = 0; k < SROUNDS; ++k) {
    const int i = tid + k * NT;
    side_kind[k] = 0;
    side_dst[k] = 0;
    side_src[k] = 0;
    if (i < NV) {
      const int ty = i / (TX / 2), pc = i % (TX / 2);
      side_kind[k] = 1;
      side_dst[k] = ty * TX + pc * 2;
      side_src[k] = tile0 + (long long)ty * B.NX + pc * 2;
    } else if (i < NV + NR) {
      const int j = i - NV, ty = j / (TX / 4), pc = j % (TX / 4);
      side_kind[k] = 2;
      side_dst[k] = ty * TX + pc * 4;
      side_src[k] = tile0 + (long long)ty * B.NX + pc * 4;
    } else if (i < NSIDE) {
      const int j = i - NV - NR, hy = j / (HX / 4), pc = j % (HX / 4);
      side_kind[k] = 3;
      side_dst[k] = hy * HX + pc * 4;
      side_src[k] = (long long)(cy0 - HAL + hy) * B.NX + (cx0 - HAL) + pc * 4;
    }
  }

  // gather one piece of a halo cell (src: load-map entry)
  auto gather = [&](int src, T *d) {
    if (src >= 0) {
      cp_async_n<COPYB>(d, in_base + src * in_ld2);
    } else if (src == -1) {
      zero_n<COPYB>(d);
    } else {
      // periodic image times the Bloch phase correction
      const int b = -(src + 2);
      const int irow = __ldg(p.per_inner + b);
      const T *g = in_base + irow * in_ld2;
      const T pr = static_cast<const T *>(p.phase_corr)[2 * b];
      const T pi = static_cast<const T *>(p.phase_corr)[2 * b + 1];
#pragma unroll
      for (int e = 0; e < COPYC; e += 2) {
        const T xr = g[e], xi = g[e + 1];
        d[e] = xr * pr - xi * pi;
        d[e + 1] = xr * pi + xi * pr;
      }
    }
  };
  // halo plane q (map in slot MS), v and rows of q, psi0 of plane q - 4
  auto load_plane = [&](int q, int DB, int RS, int MS, int RS4) {
    T *dst = reinterpret_cast<T *>(planes + DB * PLANE) + part * COPYC;
    const int *map = mapring + MS * HY * HX;
#pragma unroll
    for (int k = 0; k < HROUNDS; ++k) {
      const int cell = cell0 + k * CSTEP;
      gather(map[cell], dst + cell * SC * 2);
    }
    if (HREM && cell0 < HREM) {
      const int cell = cell0 + HROUNDS * CSTEP;
      gather(map[cell], dst + cell * SC * 2);
    }
    const long long qoff = q * planeN;
#pragma unroll
    for (int k = 0; k < SROUNDS; ++k) {
      if (side_kind[k] == 1) {
        if (p.v_cell)
          cp_async16(vring + DB * TY * TX + side_dst[k], p.v_cell + qoff + side_src[k]);
        else
          *reinterpret_cast<float4 *>(vring + DB * TY * TX + side_dst[k]) = make_float4(0.f, 0.f, 0.f, 0.f);
      } else if (side_kind[k] == 2) {
        cp_async16(rowring + RS * TY * TX + side_dst[k], p.cell_row + qoff + side_src[k]);
      }
    }
    if (X0 && q - HAL >= zs) {
      const int *ro = rowring + RS4 * TY * TX;
      T *x0d = reinterpret_cast<T *>(psi0ring + DB * INNER) + part * COPYC;
#pragma unroll
      for (int k = 0; k <= IROUNDS; ++k) {
        const int cell = cell0 + k * CSTEP;
        if (k == IROUNDS && !(IREM && cell0 < IREM)) break;
        const int row = ro[cell];
        if (row >= 0 && row < p.np) cp_async_n<COPYB>(x0d + cell * SC * 2, psi0_base + row * psi0_ld2);
      }
    }
  };
  auto load_map = [&](int q, int MS) {
#pragma unroll
    for (int k = 0; k < SROUNDS; ++k)
      if (side_kind[k] == 3) cp_async16(mapring + MS * HY * HX + side_dst[k], p.cell_src + q * planeN + side_src[k]);
  };

  // ---- weights, field, observables -------------------------------------------
  const T *w_x = wsel<T>(p.wx, p.wxf), *w_y = wsel<T>(p.wy, p.wyf), *w_z = wsel<T>(p.wz, p.wzf);
  const double fscale = p.fld_scale_dev ? *p.fld_scale_dev : 1.0;
  const double fz = p.fld[2] * fscale * B.h[2];
  double fxy[RY];
#pragma unroll
  for (int r = 0; r < RY; ++r)
    fxy[r] = fscale * (p.fld[0] * B.h[0] * double(cx0 + tx + B.lo[0]) +
                       p.fld[1] * B.h[1] * double(cy0 + tyg * RY + r + B.lo[1]));
  Kahan ke = {0, 0}, kn = {0, 0}, kd = {0, 0};

  C2 acc[RY][9];
#pragma unroll
  for (int r = 0; r < RY; ++r)
#pragma unroll
    for (int k = 0; k < 9; ++k) acc[r][k] = czero<C2>();

  // ---- prologue ---------------------------------------------------------------
  // maps of planes zbeg, zbeg+1 synchronously (slots 0, 1), then the planes
  // themselves with the maps of zbeg+2, zbeg+3 (slots 2, 0)
  for (int i = tid; i < 2 * HY * HX; i += NT) {
    const int k = i / (HY * HX), c = i - k * (HY * HX);
    const int hy = c / HX, hx = c - hy * HX;
    const int q = min(zbeg + k, zend - 1);
    mapring[k * HY * HX + c] = __ldg(p.cell_src + q * planeN + (long long)(cy0 - HAL + hy) * B.NX + cx0 - HAL + hx);
  }
  __syncthreads();
  load_plane(zbeg, 0, 0, 0, 0);
  if (zbeg + 2 < zend) load_map(zbeg + 2, 2);
  cp_async_commit();
  __syncthreads();  // everyone has read map slot 0 before it is refilled
  if (zbeg + 1 < zend) load_plane(zbeg + 1, 1, 1, 1, 0);
  if (zbeg + 3 < zend) load_map(zbeg + 3, 0);
  cp_async_commit();

  C2 *out = static_cast<C2 *>(p.out);
  const long long out_ldc = p.out_ld;
  const int cidx = chunk * SC + cs;  // complex column of this thread in a row
  const T are = static_cast<T>(p.a_re), aim = static_cast<T>(p.a_im);
  const double xr = double(cx0 + tx + B.lo[0]);

  // one plane; K = (pz - zbeg) % 9 makes every ring index static
  auto plane = [&](auto Kc, int pz) {
    constexpr int K = decltype(Kc)::value;
    constexpr int DB = K % NBUF;                       // data / v / psi0 buffer of pz
    cp_async_wait<1>();
    __syncthreads();
    if (pz + 2 < zend) load_plane(pz + 2, (K + 2) % NBUF, (K + 2) % RING, (K + 2) % NBUF, (K + 7) % RING);
    if (pz + 4 < zend) load_map(pz + 4, (K + 1) % NBUF);
    cp_async_commit();

    const C2 *P = planes + DB * PLANE;
    const double *vd = vring + DB * TY * TX;
    const double vz = fz * double(pz + B.lo[2]);

    // y arms streamed down the column (value i feeds row r with w_y[i - r]),
    // the centre carries w_c + v and the z arms; x arms after
    C2 ya[RY], yb[RY], xa[RY], xb[RY];
#pragma unroll
    for (int r = 0; r < RY; ++r) ya[r] = yb[r] = xa[r] = xb[r] = czero<C2>();
#pragma unroll
    for (int i = 0; i < RY + 8; ++i) {
      const C2 val = P[((tyg * RY + i) * HX + tx + HAL) * SC + cs];
#pragma unroll
      for (int r = 0; r < RY; ++r) {
        const int d = i - r;
        if (d < 0 || d > 8) continue;
        if (d < 4) {
          ya[r] = cfma(w_y[d], val, ya[r]);
        } else if (d > 4) {
          yb[r] = cfma(w_y[d], val, yb[r]);
        } else {
          const double vv = vd[(tyg * RY + r) * TX + tx] + fxy[r] + vz;
          xa[r] = cfma(w_x[4] + static_cast<T>(vv), val, xa[r]);
#pragma unroll
          for (int j = 0; j < 9; ++j)
            if (j != 4) acc[r][(j + K) % 9] = cfma(w_z[8 - j], val, acc[r][(j + K) % 9]);
        }
      }
    }
    C2 done[RY];
#pragma unroll
    for (int r = 0; r < RY; ++r) {
      const C2 *rp = P + ((tyg * RY + r + HAL) * HX + tx + HAL) * SC + cs;
#pragma unroll
      for (int d = -4; d <= -1; ++d) xa[r] = cfma(w_x[d + 4], rp[d * SC], xa[r]);
#pragma unroll
      for (int d = 1; d <= 4; ++d) xb[r] = cfma(w_x[d + 4], rp[d * SC], xb[r]);
      C2 &a4 = acc[r][(4 + K) % 9];
      a4.x += (ya[r].x + yb[r].x) + (xa[r].x + xb[r].x);
      a4.y += (ya[r].y + yb[r].y) + (xa[r].y + xb[r].y);
      done[r] = acc[r][K];
      acc[r][K] = czero<C2>();
    }

    // ---- outputs of plane zo = pz - 4 are complete ----------------------------
    const int zo = pz - HAL;
    if (zo >= zs) {
      const int *ro = rowring + ((K + 5) % RING) * TY * TX;
      [[maybe_unused]] const C2 *x0s = psi0ring + DB * INNER;
#pragma unroll
      for (int r = 0; r < RY; ++r) {
        const int ty = tyg * RY + r;
        const int row = ro[ty * TX + tx];
        if (row < 0 || row >= p.np) continue;
        const C2 h = done[r];
        C2 val = h;
        if constexpr (X0) {
          const C2 x0 = x0s[(ty * TX + tx) * SC + cs];
          if constexpr (OBS) {
            const double rr = p.obs_pol[0] * B.h[0] * xr + p.obs_pol[1] * B.h[1] * double(cy0 + ty + B.lo[1]) +
                              p.obs_pol[2] * B.h[2] * double(zo + B.lo[2]);
            const double n2 = double(x0.x) * double(x0.x) + double(x0.y) * double(x0.y);
            kadd(ke, double(x0.x) * double(h.x) + double(x0.y) * double(h.y));
            kadd(kn, n2);
            kadd(kd, n2 * rr);
          }
          if constexpr (HORNER) {
            val.x = x0.x + are * h.x - aim * h.y;
            val.y = x0.y + are * h.y + aim * h.x;
          }
        }
        out[row * out_ldc + cidx] = val;
      }
    }
  };

#pragma unroll 1
  for (int pz = zbeg; pz < zend; pz += 9) {
    plane(std::integral_constant<int, 0>{}, pz);
    if (pz + 1 < zend) plane(std::integral_constant<int, 1>{}, pz + 1);
    if (pz + 2 < zend) plane(std::integral_constant<int, 2>{}, pz + 2);
    if (pz + 3 < zend) plane(std::integral_constant<int, 3>{}, pz + 3);
    if (pz + 4 < zend) plane(std::integral_constant<int, 4>{}, pz + 4);
    if (pz + 5 < zend) plane(std::integral_constant<int, 5>{}, pz + 5);
    if (pz + 6 < zend) plane(std::integral_constant<int, 6>{}, pz + 6);
    if (pz + 7 < zend) plane(std::integral_constant<int, 7>{}, pz + 7);
    if (pz + 8 < zend) plane(std::integral_constant<int, 8>{}, pz + 8);
  }
  cp_async_wait<0>();

  if constexpr (OBS) {
    __syncthreads();
    double *red = reinterpret_cast<double *>(smem);  // NT x 6 doubles
    red[tid * 6 + 0] = ke.s;
    red[tid * 6 + 1] = ke.c;
    red[tid * 6 + 2] = kn.s;
    red[tid * 6 + 3] = kn.c;
    red[tid * 6 + 4] = kd.s;
    red[tid * 6 + 5] = kd.c;
    __syncthreads();
    if (tid < SC) {
      Kahan a[3] = {{0, 0}, {0, 0}, {0, 0}};
      for (int t = tid; t < NT; t += SC) {
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          kadd(a[q], red[t * 6 + 2 * q]);
          a[q].c += red[t * 6 + 2 * q + 1];
        }
      }
      double *o = p.obs + ((long long)item * p.obs_ld + chunk * SC + tid) * 6;
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        o[2 * q] = a[q].s;
        o[2 * q + 1] = a[q].c;
      }
    }
  }
}

// One system: the chunks of a work item are adjacent in launch order, so they
// run together and share each row's DRAM lines, the cell maps and v in L2.
template <typename T, int SC, int TX, int TY, int RY, bool HORNER, bool OBS>
__global__ void __launch_bounds__(SC * TX * (TY / RY), 1) pass_kernel(const __grid_constant__ PassArgs p) {
  extern __shared__ __align__(16) unsigned char smem[];
  pass_body<T, SC, TX, TY, RY, HORNER, OBS>(p, blockIdx.x / p.chunks, blockIdx.x % p.chunks, smem);
}

// Many systems in one persistent launch: each CTA takes (system, item,
// chunk) units from a list sorted by cost until it is exhausted.
template <typename T, int SC, int TX, int TY, int RY, bool HORNER>
__global__ void __launch_bounds__(SC * TX * (TY / RY), 1) pass_group_kernel(const __grid_constant__ GroupArgs g) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int unit_s;
  for (;;) {
    if (threadIdx.x == 0) unit_s = atomicAdd(g.counter, 1);
    __syncthreads();
    const int u = unit_s;
    __syncthreads();
    if (u >= g.nunits) break;
    const int4 U = g.units[u];  // {system, item, chunk, -}
    pass_body<T, SC, TX, TY, RY, HORNER, false>(g.sys[U.x], U.y, U.z, smem);
    __syncthreads();
  }
}

template <typename T, int SC, int TX, int TY, int RY, bool HORNER, bool OBS>
hpsi_status launch_mode(const PassArgs &a, cudaStream_t st) {
  using LY = PassLayout<T, SC, TX, TY, RY>;
  const size_t red = size_t(LY::NT) * 6 * sizeof(double);
  const size_t bytes = std::max(LY::bytes, red);
  auto kern = pass_kernel<T, SC, TX, TY, RY, HORNER, OBS>;
  static bool attr_set = false;
  if (!attr_set) {
    HPSI_TRY_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
    attr_set = true;
  }
  const unsigned nblocks = unsigned(a.nitems) * a.chunks;
  kern<<<nblocks, LY::NT, bytes, st>>>(a);
  HPSI_CHECK_LAUNCH();
  return HPSI_OK;
}

template <typename T, int SC, int TX, int TY, int RY>
hpsi_status launch_variant(const PassArgs &a, cudaStream_t st) {
  const bool horner = a.mode == PASS_HORNER, obs = a.obs != nullptr;
  if (horner && obs) return launch_mode<T, SC, TX, TY, RY, true, true>(a, st);
  if (horner) return launch_mode<T, SC, TX, TY, RY, true, false>(a, st);
  if (obs) return launch_mode<T, SC, TX, TY, RY, false, true>(a, st);
  return launch_mode<T, SC, TX, TY, RY, false, false>(a, st);
}

}  // namespace

// Instantiated variants (tile 16 x 16 cells): FP64 threads keep RY = 2 rows of
// 9 complex running sums, FP32 threads RY = 4.
template <typename T>
hpsi_status launch_pass(PassArgs a, const PassShape &s, cudaStream_t st) {
  if (a.nitems == 0) return HPSI_OK;
  if (s.tx == 16 && s.ty == 16) {
    if constexpr (sizeof(T) == 8) {
      if (s.ry == 2) {
        if (s.sc == 4) return launch_variant<T, 4, 16, 16, 2>(a, st);
        if (s.sc == 2) return launch_variant<T, 2, 16, 16, 2>(a, st);
        if (s.sc == 1) return launch_variant<T, 1, 16, 16, 2>(a, st);
      }
    } else {
      if (s.ry == 4) {
        if (s.sc == 8) return launch_variant<T, 8, 16, 16, 4>(a, st);
        if (s.sc == 4) return launch_variant<T, 4, 16, 16, 4>(a, st);
        if (s.sc == 2) return launch_variant<T, 2, 16, 16, 4>(a, st);
        if (s.sc == 1) return launch_variant<T, 1, 16, 16, 4>(a, st);
      }
    }
  }
  set_error("launch_pass: no kernel variant for this shape");
  return HPSI_ERR_UNSUPPORTED;
}

template <typename T, int SC, int RY>
hpsi_status launch_group_v(const GroupArgs &g, int grid, cudaStream_t st) {
  using LY = PassLayout<T, SC, 16, 16, RY>;
  const size_t bytes = LY::bytes;
  if (g.sys[0].mode == PASS_HORNER) {
    auto kern = pass_group_kernel<T, SC, 16, 16, RY, true>;
    static bool set = false;
    if (!set) {
      HPSI_TRY_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
      set = true;
    }
    kern<<<grid, LY::NT, bytes, st>>>(g);
  } else {
    auto kern = pass_group_kernel<T, SC, 16, 16, RY, false>;
    static bool set = false;
    if (!set) {
      HPSI_TRY_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
      set = true;
    }
    kern<<<grid, LY::NT, bytes, st>>>(g);
  }
  HPSI_CHECK_LAUNCH();
  return HPSI_OK;
}

template <typename T>
hpsi_status launch_pass_group(const GroupArgs &g, int sc, int num_sms, cudaStream_t st) {
  if (g.nunits == 0) return HPSI_OK;
  const int grid = std::min(g.nunits, num_sms);
  if constexpr (sizeof(T) == 8) {
    if (sc == 4) return launch_group_v<T, 4, 2>(g, grid, st);
    if (sc == 2) return launch_group_v<T, 2, 2>(g, grid, st);
    if (sc == 1) return launch_group_v<T, 1, 2>(g, grid, st);
  } else {
    if (sc == 8) return launch_group_v<T, 8, 4>(g, grid, st);
    if (sc == 4) return launch_group_v<T, 4, 4>(g, grid, st);
    if (sc == 2) return launch_group_v<T, 2, 4>(g, grid, st);
    if (sc == 1) return launch_group_v<T, 1, 4>(g, grid, st);
  }
  set_error("launch_pass_group: no kernel variant for this state chunk");
  return HPSI_ERR_UNSUPPORTED;
}

template hpsi_status launch_pass_group<double>(const GroupArgs &, int, int, cudaStream_t);
template hpsi_status launch_pass_group<float>(const GroupArgs &, int, int, cudaStream_t);
template hpsi_status launch_pass<double>(PassArgs, const PassShape &, cudaStream_t);
template hpsi_status launch_pass<float>(PassArgs, const PassShape &, cudaStream_t);

}  // namespace hpsi
