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
// sum of output p-4 is then complete and is written out after the KB ket
// term and, for a Taylor pass, the Horner update psi0 + a * H u.
//
// Reference semantics: X(nl_operator_operate_batch)
// (src/grid/nl_operator_inc.F90:21-130) with weights op%w * (-1/2),
// X(hamiltonian_elec_base_local_sub) (src/hamiltonian/hamiltonian_elec_base_inc.F90:233-242),
// the projector ket (:909-1027) and the Taylor axpys
// (src/electrons/exponential.F90:738-746).  Sums are taken in a different
// order than the reference's (rounding differences at the 1e-16 level).
#include <algorithm>
#include <cstdio>

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

template <typename T, int SC, int TX, int TY, int RY, int NBUF>
struct PassLayout {
  static constexpr int L = 2 * SC;
  static constexpr int HAL = 4;
  static constexpr int HX = TX + 2 * HAL, HY = TY + 2 * HAL;
  static constexpr int NT = L * TX * (TY / RY);
  static constexpr int PLANE = HY * HX * L;  // T elements of one halo plane
  static constexpr int INNER = TY * TX * L;  // T elements of one interior plane
  static constexpr int RING = 8;             // row ring (>= NBUF + 4)
  static constexpr int MAPS = 4;             // map ring (>= NBUF + 1)
  // byte offsets of the shared-memory regions
  static constexpr size_t off_planes = 0;
  static constexpr size_t off_psi0 = off_planes + size_t(NBUF) * PLANE * sizeof(T);
  static constexpr size_t off_v = off_psi0 + size_t(NBUF) * INNER * sizeof(T);
  static constexpr size_t off_rows = off_v + size_t(NBUF) * TY * TX * sizeof(double);
  static constexpr size_t off_maps = off_rows + size_t(RING) * TY * TX * sizeof(int);
  static constexpr size_t bytes = off_maps + size_t(MAPS) * HY * HX * sizeof(int);
};

template <typename T, int SC, int TX, int TY, int RY, int NBUF>
__global__ void __launch_bounds__(2 * SC * TX * (TY / RY), 1)
    pass_kernel(const PassArgs p) {
  using LY = PassLayout<T, SC, TX, TY, RY, NBUF>;
  constexpr int L = LY::L, HAL = LY::HAL, HX = LY::HX, HY = LY::HY, NT = LY::NT;
  constexpr int PLANE = LY::PLANE, INNER = LY::INNER, RING = LY::RING, MAPS = LY::MAPS;
  constexpr int CELLB = L * int(sizeof(T));     // bytes per cell chunk
  constexpr int COPYB = CELLB >= 16 ? 16 : CELLB;
  constexpr int CPC = CELLB / COPYB;            // copies per cell
  constexpr int COPYE = COPYB / int(sizeof(T)); // T elements per copy
  static_assert(NBUF + 4 <= RING && NBUF + 1 <= MAPS, "ring too small");
  static_assert((HX * 4) % 16 == 0 && (TX * 4) % 16 == 0, "tile rows must be 16-byte multiples");

  extern __shared__ __align__(16) unsigned char smem[];
  T *planes = reinterpret_cast<T *>(smem + LY::off_planes);
  T *psi0ring = reinterpret_cast<T *>(smem + LY::off_psi0);
  double *vring = reinterpret_cast<double *>(smem + LY::off_v);
  int *rowring = reinterpret_cast<int *>(smem + LY::off_rows);
  int *mapring = reinterpret_cast<int *>(smem + LY::off_maps);

  const int tid = threadIdx.x;
  const int lane = tid % L;
  const int tx = (tid / L) % TX;
  const int tyg = tid / (L * TX);
  // chunks of the same tile are adjacent in launch order, so they run
  // together and share each row's DRAM lines, the cell maps and v in L2
  const int chunk = blockIdx.x % p.chunks;
  const int rest = blockIdx.x / p.chunks;
  const int ntiles = p.tiles_x * p.tiles_y;
  const int tile = rest % ntiles, zblk = rest / ntiles;
  const int bx = tile % p.tiles_x, by = tile / p.tiles_x;
  const CellBox &B = p.box;
  const int cx0 = HAL + bx * TX, cy0 = HAL + by * TY;
  const int zs = HAL + zblk * p.zb;
  const int ze = min(zs + p.zb, HAL + B.nzo);
  const long long planeN = (long long)B.NX * B.NY;
  const int zbeg = zs - HAL, zend = ze + HAL;  // planes [zbeg, zend)

  const T *in = static_cast<const T *>(p.in);
  const long long in_ld2 = 2 * p.in_ld;
  const int s_off = chunk * L;
  const T *psi0 = static_cast<const T *>(p.psi0);
  const long long psi0_ld2 = 2 * p.psi0_ld;
  const bool need_x0 = psi0 != nullptr;

  // ---- asynchronous loaders -------------------------------------------------
  // halo-plane cell map of plane q (HY rows of HX ints, 16-byte pieces)
  auto load_map = [&](int q) {
    int *dst = mapring + (q & (MAPS - 1)) * HY * HX;
    const int *src = p.cell_src + q * planeN + (long long)(cy0 - HAL) * B.NX + (cx0 - HAL);
    constexpr int PER_ROW = HX / 4;
    for (int i = tid; i < HY * PER_ROW; i += NT) {
      const int hy = i / PER_ROW, part = i - hy * PER_ROW;
      cp_async16(dst + hy * HX + part * 4, src + (long long)hy * B.NX + part * 4);
    }
  };
  // gathered halo plane q (map already resident), interior v and rows of q,
  // and the pointwise psi0 values of the plane q - 4 emitted later
  auto load_plane = [&](int q) {
    const int buf = q % NBUF;
    T *dst = planes + buf * PLANE;
    const int *map = mapring + (q & (MAPS - 1)) * HY * HX;
    for (int i = tid; i < HY * HX * CPC; i += NT) {
      const int cell = i / CPC, part = i - cell * CPC;
      const int src = map[cell];
      T *d = dst + cell * L + part * COPYE;
      if (src >= 0) {
        cp_async_n<COPYB>(d, in + src * in_ld2 + s_off + part * COPYE);
      } else if (src == -1) {
        zero_n<COPYB>(d);
      } else {
        // periodic image times the Bloch phase correction
        const int b = -(src + 2);
        const int irow = __ldg(p.per_inner + b);
        const T *g = in + irow * in_ld2 + s_off + part * COPYE;
        const T pr = static_cast<const T *>(p.phase_corr)[2 * b];
        const T pi = static_cast<const T *>(p.phase_corr)[2 * b + 1];
#pragma unroll
        for (int e = 0; e < COPYE; e += 2) {
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
      T *x0d = psi0ring + buf * INNER;
      for (int i = tid; i < TY * TX * CPC; i += NT) {
        const int cell = i / CPC, part = i - cell * CPC;
        const int row = ro[cell];
        T *d = x0d + cell * L + part * COPYE;
        if (row >= 0 && row < p.np)
          cp_async_n<COPYB>(d, psi0 + row * psi0_ld2 + s_off + part * COPYE);
      }
    }
  };

  // ---- weights and field ---------------------------------------------------
  T w_x[9], w_y[9], w_z[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    w_x[k] = static_cast<T>(p.wx[k]);
    w_y[k] = static_cast<T>(p.wy[k]);
    w_z[k] = static_cast<T>(p.wz[k]);
  }
  double fscale = p.fld_scale_dev ? *p.fld_scale_dev : 1.0;
  const double fx = p.fld[0] * fscale * B.h[0], fy = p.fld[1] * fscale * B.h[1],
               fz = p.fld[2] * fscale * B.h[2];
  const bool obs_on = p.obs != nullptr;
  const double px = p.obs_pol[0] * B.h[0], py = p.obs_pol[1] * B.h[1], pzc = p.obs_pol[2] * B.h[2];

  T acc[RY][9];
#pragma unroll
  for (int r = 0; r < RY; ++r)
#pragma unroll
    for (int k = 0; k < 9; ++k) acc[r][k] = T(0);

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

  T *out = static_cast<T *>(p.out);
  const long long out_ld2 = 2 * p.out_ld;
  const T *kb_pt = static_cast<const T *>(p.kb_pt);
  const T *projv = static_cast<const T *>(p.proj);
  const long long proj_ld2 = 2 * p.proj_ld;

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
    const T *P = planes + buf * PLANE;
    const double *vd = vring + buf * TY * TX;

    // y window of this thread's column
    T col[RY + 8];
#pragma unroll
    for (int i = 0; i < RY + 8; ++i) col[i] = P[((tyg * RY + i) * HX + tx + HAL) * L + lane];

    const double xr = double(cx0 + tx + B.lo[0]);
    const double zr = double(pz + B.lo[2]);
#pragma unroll
    for (int r = 0; r < RY; ++r) {
      const T c = col[r + 4];
#pragma unroll
      for (int k = 0; k < 9; ++k)
        if (k != 4) acc[r][k] += w_z[8 - k] * c;
      T s = acc[r][4];
#pragma unroll
      for (int d = -4; d <= 4; ++d)
        if (d != 0) s += w_y[d + 4] * col[r + 4 + d];
      const T *rp = P + ((tyg * RY + r + HAL) * HX + tx + HAL) * L + lane;
#pragma unroll
      for (int d = -4; d <= 4; ++d)
        if (d != 0) s += w_x[d + 4] * rp[d * L];
      const int ty = tyg * RY + r;
      const double yr = double(cy0 + ty + B.lo[1]);
      const double vv = vd[ty * TX + tx] + fx * xr + fy * yr + fz * zr;
      s += (w_x[4] + static_cast<T>(vv)) * c;
      acc[r][4] = s;
    }

    // ---- epilogue: outputs of plane zo = pz - 4 are complete ---------------
    const int zo = pz - HAL;
    if (zo >= zs) {
      const int *ro = rowring + (zo & (RING - 1)) * TY * TX;
      const T *x0s = psi0ring + buf * INNER;
#pragma unroll
      for (int r = 0; r < RY; ++r) {
        const int ty = tyg * RY + r;
        const int rowv = ro[ty * TX + tx];
        const int row = (rowv >= 0 && rowv < p.np) ? rowv : -1;
        T h = acc[r][0];
        if (row >= 0 && p.kb_ptr) {
          const int e0 = __ldg(p.kb_ptr + row), e1 = __ldg(p.kb_ptr + row + 1);
          for (int e = e0; e < e1; ++e) {
            const int4 E = __ldg(p.kb_ent + e);
            const T *pt = kb_pt + E.x;
            const T *pr = projv + (long long)E.y * proj_ld2 + s_off + lane;
            for (int j = 0; j < E.z; ++j) h += pt[j] * pr[j * proj_ld2];
          }
        }
        const T partner = __shfl_xor_sync(0xffffffffu, h, 1);
        const T x0 = need_x0 ? x0s[(ty * TX + tx) * L + lane] : T(0);
        if (obs_on && row >= 0) {
          const double xd = double(x0);
          const double rr = px * xr + py * double(cy0 + ty + B.lo[1]) + pzc * double(zo + B.lo[2]);
          kadd(ke, xd * double(h));
          kadd(kn, xd * xd);
          kadd(kd, xd * xd * rr);
        }
        if (row >= 0) {
          T val;
          if (p.mode == PASS_HORNER) {
            const T are = static_cast<T>(p.a_re), aim = static_cast<T>(p.a_im);
            if ((lane & 1) == 0)
              val = x0 + are * h - aim * partner;  // real part
            else
              val = x0 + are * h + aim * partner;  // imaginary part
          } else {
            val = h;
          }
          out[row * out_ld2 + s_off + lane] = val;
        }
      }
    }
#pragma unroll
    for (int r = 0; r < RY; ++r) {
#pragma unroll
      for (int k = 0; k < 8; ++k) acc[r][k] = acc[r][k + 1];
      acc[r][8] = T(0);
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
      const int s = tid;
      Kahan a[3] = {{0, 0}, {0, 0}, {0, 0}};
      for (int t = 0; t < NT; ++t) {
        const int ln = t % L;
        if ((ln >> 1) != s) continue;
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          kadd(a[q], red[t * 6 + 2 * q]);
          a[q].c += red[t * 6 + 2 * q + 1];
        }
      }
      const int cta = tile + ntiles * zblk;
      double *o = p.obs + ((long long)cta * p.obs_ld + chunk * SC + s) * 6;
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
  const unsigned nblocks = unsigned(a.tiles_x) * a.tiles_y * a.zblocks * a.chunks;
  kern<<<nblocks, LY::NT, bytes, st>>>(a);
  HPSI_CHECK_LAUNCH();
  return HPSI_OK;
}

}  // namespace

void pass_geometry(PassArgs &a, const PassShape &s, int ld, int num_sms) {
  const CellBox &B = a.box;
  a.tiles_x = (B.nxo + s.tx - 1) / s.tx;
  a.tiles_y = (B.nyo + s.ty - 1) / s.ty;
  a.chunks = ld / s.sc;
  // z blocks: enough CTAs for ~4 waves while keeping the z halo overhead small
  const long long base = (long long)a.tiles_x * a.tiles_y * a.chunks;
  int zb = B.nzo;
  const long long want = 4LL * num_sms;
  while (zb > 16 && base * ((B.nzo + zb - 1) / zb) < want) zb = (zb + 1) / 2;
  a.zb = zb;
  a.zblocks = (B.nzo + zb - 1) / zb;
}

template <typename T, int TX, int TY, int RY>
hpsi_status launch_sc(const PassArgs &a, int sc, cudaStream_t st) {
  switch (sc) {
    case 1:
      return launch_variant<T, 1, TX, TY, RY>(a, st);
    case 2:
      return launch_variant<T, 2, TX, TY, RY>(a, st);
    case 4:
      return launch_variant<T, 4, TX, TY, RY>(a, st);
    case 8:
      if constexpr (sizeof(T) == 4) return launch_variant<T, 8, TX, TY, RY>(a, st);
      break;
  }
  set_error("launch_pass: no kernel variant for this state chunk");
  return HPSI_ERR_UNSUPPORTED;
}

template <typename T>
hpsi_status launch_pass(PassArgs a, const PassShape &s, cudaStream_t st) {
  if (s.tx == 16 && s.ty == 16 && s.ry == 4) return launch_sc<T, 16, 16, 4>(a, s.sc, st);
  if (s.tx == 16 && s.ty == 16 && s.ry == 8) return launch_sc<T, 16, 16, 8>(a, s.sc, st);
  set_error("launch_pass: no kernel variant for this shape");
  return HPSI_ERR_UNSUPPORTED;
}

template hpsi_status launch_pass<double>(PassArgs, const PassShape &, cudaStream_t);
template hpsi_status launch_pass<float>(PassArgs, const PassShape &, cudaStream_t);

}  // namespace hpsi
