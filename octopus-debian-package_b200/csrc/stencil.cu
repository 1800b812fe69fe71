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

template <typename T, int SC, int TX, int TY, int RY, int NBUF>
struct PassLayout {
  using C2 = typename Cx<T>::type;
  static constexpr int HAL = 4;
  static constexpr int HX = TX + 2 * HAL, HY = TY + 2 * HAL;
  static constexpr int NT = SC * TX * (TY / RY);
  static constexpr int PLANE = HY * HX * SC;  // complex numbers of one halo plane
  static constexpr int INNER = TY * TX * SC;  // complex numbers of one interior plane
  static constexpr int RING = 8;              // row ring (>= NBUF + 4)
  static constexpr int MAPS = 4;              // map ring (>= NBUF + 1)
  // byte offsets of the shared-memory regions
  static constexpr size_t off_planes = 0;
  static constexpr size_t off_psi0 = off_planes + size_t(NBUF) * PLANE * sizeof(C2);
  static constexpr size_t off_v = off_psi0 + size_t(NBUF) * INNER * sizeof(C2);
  static constexpr size_t off_rows = off_v + size_t(NBUF) * TY * TX * sizeof(double);
  static constexpr size_t off_maps = off_rows + size_t(RING) * TY * TX * sizeof(int);
  static constexpr size_t bytes = off_maps + size_t(MAPS) * HY * HX * sizeof(int);
};

// Each thread owns one complex state (re and im together) of RY consecutive
// y cells of one x column; a warp reads whole contiguous cell chunks.
template <typename T, int SC, int TX, int TY, int RY, int NBUF>
__global__ void __launch_bounds__(SC * TX * (TY / RY), 1)
    pass_kernel(const PassArgs p) {
  using LY = PassLayout<T, SC, TX, TY, RY, NBUF>;
  using C2 = typename LY::C2;
  constexpr int HAL = LY::HAL, HX = LY::HX, HY = LY::HY, NT = LY::NT;
  constexpr int PLANE = LY::PLANE, INNER = LY::INNER, RING = LY::RING, MAPS = LY::MAPS;
  constexpr int CELLB = SC * int(sizeof(C2));   // bytes per cell chunk
  constexpr int COPYB = CELLB >= 16 ? 16 : CELLB;
  constexpr int CPC = CELLB / COPYB;            // copies per cell
  constexpr int COPYC = COPYB / int(sizeof(T)); // T elements per copy
  static_assert(NBUF + 4 <= RING && NBUF + 1 <= MAPS, "ring too small");

  extern __shared__ __align__(16) unsigned char smem[];
  C2 *planes = reinterpret_cast<C2 *>(smem + LY::off_planes);
  C2 *psi0ring = reinterpret_cast<C2 *>(smem + LY::off_psi0);
  double *vring = reinterpret_cast<double *>(smem + LY::off_v);
  int *rowring = reinterpret_cast<int *>(smem + LY::off_rows);
  int *mapring = reinterpret_cast<int *>(smem + LY::off_maps);

  const int tid = threadIdx.x;
  const int cs = tid % SC;              // complex state within the chunk
  const int tx = (tid / SC) % TX;
  const int tyg = tid / (SC * TX);
  // one work item = one tile column over a z range that holds inner points;
  // the chunks of an item are adjacent in launch order, so they run together
  // and share each row's DRAM lines, the cell maps and v in L2
  const int chunk = blockIdx.x % p.chunks;
  const int item = blockIdx.x / p.chunks;
  const int4 it = p.items[item];
  const CellBox &B = p.box;
  const int cx0 = HAL + it.x * TX, cy0 = HAL + it.y * TY;
  const int zs = it.z, ze = it.w;
  const long long planeN = (long long)B.NX * B.NY;
  const int zbeg = zs - HAL, zend = ze + HAL;  // planes [zbeg, zend)

  const T *in = static_cast<const T *>(p.in);
  const long long in_ld2 = 2 * p.in_ld;
  const int s_off = chunk * SC * 2;  // T offset of this chunk within a row
  const T *psi0 = static_cast<const T *>(p.psi0);
  const long long psi0_ld2 = 2 * p.psi0_ld;
  const bool need_x0 = psi0 != nullptr;

  // ---- asynchronous loaders -------------------------------------------------
  auto load_map = [&](int q) {
    int *dst = mapring + (q & (MAPS - 1)) * HY * HX;
    const int *src = p.cell_src + q * planeN + (long long)(cy0 - HAL) * B.NX + (cx0 - HAL);
    constexpr int PER_ROW = HX / 4;
    for (int i = tid; i < HY * PER_ROW; i += NT) {
      const int hy = i / PER_ROW, part = i - hy * PER_ROW;
      cp_async16(dst + hy * HX + part * 4, src + (long long)hy * B.NX + part * 4);
    }
  };
  auto load_plane = [&](int q) {
    const int buf = q % NBUF;
    T *dst = reinterpret_cast<T *>(planes + buf * PLANE);
    const int *map = mapring + (q & (MAPS - 1)) * HY * HX;
    // thread t always copies piece t % CPC of its cells (coalesced: the CPC
    // pieces of a cell chunk are adjacent threads)
    for (int cell = tid / CPC, part = tid % CPC; cell < HY * HX; cell += NT / CPC) {
      const int src = map[cell];
      T *d = dst + cell * SC * 2 + part * COPYC;
      if (src >= 0) {
        cp_async_n<COPYB>(d, in + src * in_ld2 + s_off + part * COPYC);
      } else if (src == -1) {
        zero_n<COPYB>(d);
      } else {
        // periodic image times the Bloch phase correction
        const int b = -(src + 2);
        const int irow = __ldg(p.per_inner + b);
        const T *g = in + irow * in_ld2 + s_off + part * COPYC;
        const T pr = static_cast<const T *>(p.phase_corr)[2 * b];
        const T pi = static_cast<const T *>(p.phase_corr)[2 * b + 1];
#pragma unroll
        for (int e = 0; e < COPYC; e += 2) {
          const T xr = g[e], xi = g[e + 1];
          d[e] = xr * pr - xi * pi;
          d[e + 1] = xr * pi + xi * pr;
        }
      }
    }
    double *vd = vring + buf * TY * TX;
    int *rd = rowring + (q & (RING - 1)) * TY * TX;
    const long long base = q * planeN + (long long)cy0 * B.NX + cx0;
    for (int i = tid; i < TY * (TX / 2); i += NT) {  // v: 2 doubles per copy
      const int ty = i / (TX / 2), part = i - ty * (TX / 2);
      if (p.v_cell)
        cp_async16(vd + ty * TX + part * 2, p.v_cell + base + (long long)ty * B.NX + part * 2);
      else
        *reinterpret_cast<float4 *>(vd + ty * TX + part * 2) = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    for (int i = tid; i < TY * (TX / 4); i += NT) {  // rows: 4 ints per copy
      const int ty = i / (TX / 4), part = i - ty * (TX / 4);
      cp_async16(rd + ty * TX + part * 4, p.cell_row + base + (long long)ty * B.NX + part * 4);
    }
    const int qo = q - HAL;
    if (need_x0 && qo >= zs) {
      const int *ro = rowring + (qo & (RING - 1)) * TY * TX;
      T *x0d = reinterpret_cast<T *>(psi0ring + buf * INNER);
      for (int cell = tid / CPC, part = tid % CPC; cell < TY * TX; cell += NT / CPC) {
        const int rv = ro[cell];
        const int row = rv & 0x3fffffff;  // bit 30 flags rows with KB entries
        if (rv >= 0 && row < p.np)
          cp_async_n<COPYB>(x0d + cell * SC * 2 + part * COPYC, psi0 + row * psi0_ld2 + s_off + part * COPYC);
      }
    }
  };

  // ---- weights and field ---------------------------------------------------
  // weights are read straight from the kernel parameters (constant bank),
  // so they cost no registers
  const T *w_x = wsel<T>(p.wx, p.wxf), *w_y = wsel<T>(p.wy, p.wyf), *w_z = wsel<T>(p.wz, p.wzf);
  const double fscale = p.fld_scale_dev ? *p.fld_scale_dev : 1.0;
  const double fx = p.fld[0] * fscale * B.h[0], fy = p.fld[1] * fscale * B.h[1],
               fz = p.fld[2] * fscale * B.h[2];
  const bool obs_on = p.obs != nullptr;
  const double px = p.obs_pol[0] * B.h[0], py = p.obs_pol[1] * B.h[1], pzc = p.obs_pol[2] * B.h[2];

  C2 acc[RY][9];
#pragma unroll
  for (int r = 0; r < RY; ++r)
#pragma unroll
    for (int k = 0; k < 9; ++k) acc[r][k] = czero<C2>();

  Kahan ke = {0, 0}, kn = {0, 0}, kd = {0, 0};

  // ---- prologue: maps of the first NBUF-1 planes synchronously, then the
  // groups G(q) = {plane q, map of plane q+NBUF-1} for those planes
#pragma unroll 1
  for (int k = 0; k < NBUF - 1; ++k) {
    const int q = zbeg + k;
    if (q >= zend) break;
    int *dst = mapring + (q & (MAPS - 1)) * HY * HX;
    for (int i = tid; i < HY * HX; i += NT) {
      const int hy = i / HX, hx = i - hy * HX;
      dst[i] = __ldg(p.cell_src + q * planeN + (long long)(cy0 - HAL + hy) * B.NX + cx0 - HAL + hx);
    }
  }
  __syncthreads();
#pragma unroll 1
  for (int k = 0; k < NBUF - 1; ++k) {
    const int q = zbeg + k;
    if (q < zend) load_plane(q);
    if (q + NBUF - 1 < zend) load_map(q + NBUF - 1);
    cp_async_commit();
  }

  C2 *out = static_cast<C2 *>(p.out);
  const long long out_ldc = p.out_ld;
  const double xr = double(cx0 + tx + B.lo[0]);
  const int cidx = chunk * SC + cs;  // complex column of this thread in a row
  const T are = static_cast<T>(p.a_re), aim = static_cast<T>(p.a_im);
  const bool horner = p.mode == PASS_HORNER;

  int ring = 0;
#pragma unroll 1
  for (int pz = zbeg; pz < zend; ++pz) {
    cp_async_wait<NBUF - 2>();
    __syncthreads();
    {
      const int q = pz + NBUF - 1;
      if (q < zend) load_plane(q);
      if (q + NBUF - 1 < zend) load_map(q + NBUF - 1);
      cp_async_commit();
    }
    const int buf = pz % NBUF;
    const C2 *P = planes + buf * PLANE;
    const double *vd = vring + buf * TY * TX;
    const double zr = double(pz + B.lo[2]);

    // Slot (j + K) % 9 of acc holds the running sum of output plane pz - 4 + j
    // with K = (pz - zbeg) % 9, so the ring never moves; the slot of the
    // completed output pz - 4 is handed to the epilogue and cleared.
    C2 done[RY];
    auto compute = [&](auto Kc) {
      constexpr int K = decltype(Kc)::value;
      // y arms, streamed down the column: value i feeds row r with weight
      // w_y[i - r]; the centre (i - r == 4) carries w_c + v and the z arms
      C2 xy[RY];
#pragma unroll
      for (int r = 0; r < RY; ++r) xy[r] = czero<C2>();
#pragma unroll
      for (int i = 0; i < RY + 8; ++i) {
        const C2 val = P[((tyg * RY + i) * HX + tx + HAL) * SC + cs];
#pragma unroll
        for (int r = 0; r < RY; ++r) {
          const int d = i - r;  // 0..8, offset d - 4
          if (d < 0 || d > 8) continue;
          if (d != 4) {
            xy[r] = cfma(w_y[d], val, xy[r]);
          } else {
            const int ty = tyg * RY + r;
            const double yr = double(cy0 + ty + B.lo[1]);
            const double vv = vd[ty * TX + tx] + fx * xr + fy * yr + fz * zr;
            xy[r] = cfma(w_x[4] + static_cast<T>(vv), val, xy[r]);
#pragma unroll
            for (int j = 0; j < 9; ++j)
              if (j != 4) acc[r][(j + K) % 9] = cfma(w_z[8 - j], val, acc[r][(j + K) % 9]);
          }
        }
      }
      // x arms
#pragma unroll
      for (int r = 0; r < RY; ++r) {
        const C2 *rp = P + ((tyg * RY + r + HAL) * HX + tx + HAL) * SC + cs;
#pragma unroll
        for (int d = -4; d <= 4; ++d)
          if (d != 0) xy[r] = cfma(w_x[d + 4], rp[d * SC], xy[r]);
        acc[r][(4 + K) % 9].x += xy[r].x;
        acc[r][(4 + K) % 9].y += xy[r].y;
        done[r] = acc[r][K];
        acc[r][K] = czero<C2>();
      }
    };
    switch (ring) {
      case 0: compute(std::integral_constant<int, 0>{}); break;
      case 1: compute(std::integral_constant<int, 1>{}); break;
      case 2: compute(std::integral_constant<int, 2>{}); break;
      case 3: compute(std::integral_constant<int, 3>{}); break;
      case 4: compute(std::integral_constant<int, 4>{}); break;
      case 5: compute(std::integral_constant<int, 5>{}); break;
      case 6: compute(std::integral_constant<int, 6>{}); break;
      case 7: compute(std::integral_constant<int, 7>{}); break;
      default: compute(std::integral_constant<int, 8>{}); break;
    }
    ring = ring == 8 ? 0 : ring + 1;

    // ---- epilogue: outputs of plane zo = pz - 4 are complete ---------------
    const int zo = pz - HAL;
    if (zo >= zs) {
      const int *ro = rowring + (zo & (RING - 1)) * TY * TX;
      const C2 *x0s = psi0ring + buf * INNER;
#pragma unroll
      for (int r = 0; r < RY; ++r) {
        const int ty = tyg * RY + r;
        const int rowv = ro[ty * TX + tx];
        const int rr0 = rowv & 0x3fffffff;
        const int row = (rowv >= 0 && rr0 < p.np) ? rr0 : -1;
        const C2 h = done[r];
        if (row >= 0) {
          const C2 x0 = need_x0 ? x0s[(ty * TX + tx) * SC + cs] : czero<C2>();
          if (obs_on) {
            const double rr = px * xr + py * double(cy0 + ty + B.lo[1]) + pzc * double(zo + B.lo[2]);
            const double n2 = double(x0.x) * double(x0.x) + double(x0.y) * double(x0.y);
            kadd(ke, double(x0.x) * double(h.x) + double(x0.y) * double(h.y));
            kadd(kn, n2);
            kadd(kd, n2 * rr);
          }
          C2 val = h;
          if (horner) {
            val.x = x0.x + are * h.x - aim * h.y;
            val.y = x0.y + are * h.y + aim * h.x;
          }
          out[row * out_ldc + cidx] = val;
        }
      }
    }
  }
  cp_async_wait<0>();

  if (obs_on) {
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

template <typename T, int SC, int TX, int TY, int RY>
hpsi_status launch_variant(const PassArgs &a, cudaStream_t st) {
  constexpr int NBUF = 3;
  using LY = PassLayout<T, SC, TX, TY, RY, NBUF>;
  const size_t red = size_t(LY::NT) * 6 * sizeof(double);
  const size_t bytes = std::max(LY::bytes, red);
  auto kern = pass_kernel<T, SC, TX, TY, RY, NBUF>;
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

template hpsi_status launch_pass<double>(PassArgs, const PassShape &, cudaStream_t);
template hpsi_status launch_pass<float>(PassArgs, const PassShape &, cudaStream_t);

}  // namespace hpsi
