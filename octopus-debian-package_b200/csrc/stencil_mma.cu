// FP64 stencil pass with the x and y arms on the FP64 tensor cores (DMMA).
//
// Same work items, fill ring, z march and pass modes as the register-blocked
// pass (stencil_blk_impl.cuh); the in-plane part of the star is computed as
// two banded matrix products per warp instead of per-thread multiply-adds.
// A CTA of 512 threads owns a 16 x 8 cell tile and one 128-byte chunk of
// every row (8 complex states).  Warp w takes state j = w / 2 and the x half
// h = w % 2 (8 x 8 cells).  For the real and the imaginary part of that state,
// with IN the halo plane of the part and OUT[y][x] the in-plane star:
//
//   y arm:  OUT[y][x] += sum_hy Wy[y][hy] IN[hy][x]      Wy[y][hy] = wy[hy - y]
//   x arm:  OUT[y][x] += sum_hx IN[y][hx] Wx[x][hx]      Wx[x][hx] = wx[hx - x]
//
// as mma.sync.m8n8k4.f64 (M = 8 rows y, N = 8 columns x, K = 16 halo cells:
// four k steps each; the band of 9 weights fills 9 of every 16 columns).
// The centre weight rides on the y arm's diagonal.  Both products land in
// the same accumulator layout (thread: row y = lane / 4, columns
// 2 (lane % 4) + {0, 1}); column n of a tile is cell x = n / 2 + 4 (n % 2),
// so a thread owns cells x = lane % 4 and lane % 4 + 4 of its half, and
// those two accumulators are the running sums of the z march: the z arm and
// the local potential stay per-thread multiply-adds on the thread's own
// cells (9 running sums per cell and part).
//
// Shared-memory layout of a halo plane: one 16-byte piece (re, im of one
// state) per cell, the pieces of state j in their own plane of pitch
// (HC + 1) pieces, cell (hy, hx) at hy HX + (hx ^ f(hy)) with
// f(hy) = (hy & 3) | 4 (hy & 1).  A 16-byte load is served a quarter warp
// (8 threads) at a time; with f the 8 pieces a quarter warp reads (y-arm
// operand: 4 rows x cells {x, x + 4}; x-arm operand and centres: 2 rows x 4
// cells) and the 8 a quarter warp of the fill writes (one cell, 8 state
// planes) sit in 8 different groups of 4 banks: no conflict.
//
// The products are summed in another order than the per-thread pass, so
// results agree with it (and with the oracle) to rounding, not bit for bit.
//
// Reference semantics as in stencil.cu: X(nl_operator_operate_batch)
// (src/grid/nl_operator_inc.F90:21-130), the local potential
// (src/hamiltonian/hamiltonian_elec_base_inc.F90:233-242) and the Taylor
// axpys (src/electrons/exponential.F90:738-746).
#include <mutex>

#include "stencil_blk_impl.cuh"

namespace hpsi {
namespace mma {

using blk::cp_async16_zfill;
using blk::zero16;

template <bool X0>
struct Layout {
  static constexpr int NS = 8;  // complex states of a 128-byte chunk
  static constexpr int TX = 16, TY = 8, HAL = 4;
  static constexpr int HX = TX + 2 * HAL, HY = TY + 2 * HAL;
  static constexpr int HC = HX * HY, IC = TX * TY;
  static constexpr int NT = 512;
  static constexpr int SC = 2 * HAL * TX + TY * HX;  // star cells of a halo plane
  static constexpr int PCS = 8;                      // 16-byte pieces per cell chunk
  static constexpr int SROUNDS = (SC * PCS + NT - 1) / NT;
  static constexpr int IROUNDS = (IC * PCS + NT - 1) / NT;
  static_assert((SC * PCS) % NT == 0 && (IC * PCS) % NT == 0, "whole copy rounds");
  static constexpr int JP = (HC + 1) * 16;   // bytes per state plane (pitch = 1 piece mod 8)
  static constexpr int JP0 = (IC + 1) * 16;  // the same for the psi0 rows
  static constexpr int NBUF = X0 ? 3 : 4;
  static constexpr int NSIDE = 8, SIDE_AHEAD = 2 * NBUF - 2;
  static constexpr size_t o_psi0 = size_t(NS) * JP;
  static constexpr size_t o_v = o_psi0 + (X0 ? size_t(NS) * JP0 : 0);
  static constexpr size_t STAGE = o_v + size_t(IC) * sizeof(double);
  static constexpr size_t s_rows = size_t(HC) * sizeof(int);
  static constexpr size_t SIDEB = s_rows + size_t(IC) * sizeof(int);
  static constexpr size_t o_side = NBUF * STAGE;
  static constexpr size_t bytes = o_side + NSIDE * SIDEB;
  static_assert(bytes <= 232448 - 1024, "shared memory per CTA");
  static_assert(STAGE % 16 == 0 && o_psi0 % 16 == 0 && o_v % 16 == 0, "16-byte copies");
  static constexpr int NMAPP = HC / 4, NROWP = IC / 4, NVP = IC / 2;
  static_assert(NMAPP + NROWP <= NT && NVP <= NT, "one side piece per thread");
  static_assert(NSIDE >= 2 * NBUF - 1, "side slot lifetime");
};

// piece offset (in 16-byte pieces) of halo cell (hy, hx) in a state plane
__device__ __forceinline__ int halo_swz(int hy) { return (hy & 3) | ((hy & 1) << 2); }
__device__ __forceinline__ int halo_piece(int hy, int hx) { return hy * 24 + (hx ^ halo_swz(hy)); }
// the same for an interior cell (psi0 rows)
__device__ __forceinline__ int tile_piece(int y, int x) { return y * 16 + (x ^ ((y & 1) << 2)); }
// double offset of the potential of interior cell (y, x)
__device__ __forceinline__ int v_slot(int y, int x) { return y * 16 + (x ^ ((y & 3) << 2)); }
// int offset of the output row of interior cell (y, x) in a side slot (the 8
// rows a warp reads per cell column land in 8 different bank groups)
__device__ __forceinline__ int row_slot(int y, int x) { return y * 16 + (x ^ (((y >> 1) & 3) << 2)); }

// star cell of copy round j (0..4) for cell slot c (0..63) as (hy, hx): the
// rows above the tile over its columns, the tile rows over the tile columns
// (two rounds), the four cells either side of the tile rows, the rows below.
// Shifts and masks only; four consecutive slots are four consecutive cells
// of one row.
__device__ __forceinline__ int2 star_yx(int j, int c) {
  if (j == 0) return make_int2(c >> 4, 4 + (c & 15));
  if (j == 1 || j == 2) {
    const int i = c + 64 * (j - 1);
    return make_int2(4 + (i >> 4), 4 + (i & 15));
  }
  if (j == 3) {
    const int sx = c & 7;
    return make_int2(4 + (c >> 3), sx + ((sx >> 2) << 4));
  }
  return make_int2(12 + (c >> 4), 4 + (c & 15));
}

__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

template <bool HORNER, bool OBS>
__global__ void __launch_bounds__(512, 1) pass_mma_kernel(const __grid_constant__ PassArgs p) {
  constexpr bool X0 = HORNER || OBS;
  using LY = Layout<X0>;
  constexpr int TX = LY::TX, HAL = LY::HAL, HX = LY::HX, NBUF = LY::NBUF, NSIDE = LY::NSIDE;
  constexpr int SL = 16;  // doubles of a cell chunk
  extern __shared__ __align__(128) unsigned char smem[];

  const int ih = blockIdx.x / p.chunks, chunk = blockIdx.x % p.chunks;
  const CellBox &B = p.box;
  const int4 it = p.items[ih];
  const int cx0 = HAL + it.x * TX, cy0 = HAL + it.y * LY::TY;
  const int zs = it.z, ze = it.w;
  const int zbeg = zs - HAL, nplanes = ze - zs + 2 * HAL;
  const long long planeN = (long long)B.NX * B.NY;
  const int tid = threadIdx.x;
  const int col = chunk * SL;

  auto stage = [&](int k) { return smem + size_t(k % NBUF) * LY::STAGE; };
  auto side = [&](int k) { return smem + LY::o_side + size_t(k % NSIDE) * LY::SIDEB; };

  // ---- copy roles: star cell slot cpc, state piece `piece` ----------------------
  const int cpc = tid / LY::PCS, piece = tid % LY::PCS;
  __builtin_assume(cpc >= 0 && cpc < LY::NT / LY::PCS);
  static_assert(LY::NT / LY::PCS == 64 && LY::SROUNDS == 5, "star rounds of 64 cells");
  const double *in_base = static_cast<const double *>(p.in) + col + piece * 2;
  const long long in_ld2 = 2 * p.in_ld;
  const double *x0_base = static_cast<const double *>(p.psi0) + col + piece * 2;
  const long long x0_ld2 = 2 * p.psi0_ld;
  long long side_src = 0;
  int side_dst = -1, side_kind = 0;
  if (tid < LY::NMAPP) {
    const int c = 4 * tid, hy = c / HX, hx = c % HX;
    side_kind = 1;
    side_dst = c;
    side_src = (long long)(cy0 - HAL + hy) * B.NX + cx0 - HAL + hx;
  } else if (tid < LY::NMAPP + LY::NROWP) {
    const int c = 4 * (tid - LY::NMAPP);
    side_kind = 2;
    side_dst = row_slot(c / TX, c % TX);
    side_src = (long long)(cy0 + c / TX) * B.NX + cx0 + c % TX;
  }
  const int vc = 2 * tid;
  const long long v_src = (long long)(cy0 + vc / TX) * B.NX + cx0 + vc % TX;
  const int v_dst = v_slot(vc / TX, vc % TX);

  auto issue_side = [&](int k) {
    if (k >= nplanes || side_kind == 0) return;
    unsigned char *sd = side(k);
    const int q = zbeg + k;
    if (side_kind == 1) {
      cp_async16(reinterpret_cast<int *>(sd) + side_dst, p.cell_src + q * planeN + side_src);
    } else {
      int *d = reinterpret_cast<int *>(sd + LY::s_rows) + side_dst;
      if (q - HAL >= zs)
        cp_async16(d, p.cell_row + (q - HAL) * planeN + side_src);
      else
        *reinterpret_cast<int4 *>(d) = make_int4(-1, -1, -1, -1);
    }
  };
  auto issue_data = [&](int k) {
    if (k >= nplanes) return;
    unsigned char *st = stage(k);
    const int *map = reinterpret_cast<const int *>(side(k));
    double *plane_j = reinterpret_cast<double *>(st + size_t(piece) * LY::JP);
    if (p.phase_corr == nullptr) {
#pragma unroll
      for (int j = 0; j < LY::SROUNDS; ++j) {
        const int2 c = star_yx(j, cpc);
        const int src = map[c.x * HX + c.y];
        cp_async16_zfill(plane_j + 2 * halo_piece(c.x, c.y), in_base + max(src, 0) * in_ld2, src >= 0 ? 16 : 0);
      }
    } else {
#pragma unroll 1
      for (int j = 0; j < LY::SROUNDS; ++j) {
        const int2 c = star_yx(j, cpc);
        const int src = map[c.x * HX + c.y];
        double *d = plane_j + 2 * halo_piece(c.x, c.y);
        if (src >= 0) {
          cp_async16(d, in_base + src * in_ld2);
        } else if (src == -1) {
          zero16(d);
        } else {
          // periodic image times the Bloch phase correction
          const int b = -(src + 2);
          const double *g = in_base + __ldg(p.per_inner + b) * in_ld2;
          const double pr = static_cast<const double *>(p.phase_corr)[2 * b];
          const double pi = static_cast<const double *>(p.phase_corr)[2 * b + 1];
          const double xr = g[0], xi = g[1];
          d[0] = xr * pr - xi * pi;
          d[1] = xr * pi + xi * pr;
        }
      }
    }
    const int q = zbeg + k;
    if (X0 && q - HAL >= zs) {
      const int *rows = reinterpret_cast<const int *>(side(k) + LY::s_rows);
      double *x0 = reinterpret_cast<double *>(st + LY::o_psi0 + size_t(piece) * LY::JP0);
#pragma unroll
      for (int j = 0; j < LY::IROUNDS; ++j) {
        const int cell = cpc + j * (LY::NT / LY::PCS);
        const int row = rows[row_slot(cell / TX, cell % TX)];
        const bool ok = row >= 0 && row < p.np;
        cp_async16_zfill(x0 + 2 * tile_piece(cell / TX, cell % TX), x0_base + (ok ? row : 0) * x0_ld2, ok ? 16 : 0);
      }
    }
    if (tid < LY::NVP) {
      double *vd = reinterpret_cast<double *>(st + LY::o_v) + v_dst;
      if (p.v_cell)
        cp_async16(vd, p.v_cell + q * planeN + v_src);
      else
        zero16(vd);
    }
  };

  // ---- prologue (as the blocked pass) ----------------------------------------------
  for (int k = 0; k < NBUF - 1 && k < nplanes; ++k) {
    unsigned char *sd = side(k);
    const int q = zbeg + k;
    for (int i = tid; i < LY::HC; i += LY::NT) {
      const int hy = i / HX, hx = i % HX;
      reinterpret_cast<int *>(sd)[i] = __ldg(p.cell_src + q * planeN + (long long)(cy0 - HAL + hy) * B.NX + cx0 - HAL + hx);
    }
    for (int i = tid; i < LY::IC; i += LY::NT)
      reinterpret_cast<int *>(sd + LY::s_rows)[row_slot(i / TX, i % TX)] =
          q - HAL >= zs ? __ldg(p.cell_row + (q - HAL) * planeN + (long long)(cy0 + i / TX) * B.NX + cx0 + i % TX)
                        : -1;
  }
  __syncthreads();
  for (int k = 0; k < NBUF - 1; ++k) {
    issue_data(k);
    issue_side(k + NBUF - 1);
    cp_async_commit();
  }

  // ---- compute roles ---------------------------------------------------------------
  const int warp = tid >> 5, ln = tid & 31;
  const int js = warp >> 1, hh = warp & 1;  // state of the chunk, x half of the tile
  const int r = ln >> 2, cq = ln & 3;       // fragment row (cell y), column pair
  const int xa = 8 * hh + cq, xb = xa + 4;  // the thread's cells (tile x), row y = r
  const int pr = r & 1;
  // weight fragments: y arm A[m = r][k = 4 ks + cq] = wy[4 ks + cq - r] (centre
  // weight on the diagonal); x arm B[k = 4 ks + cq][n = r] = wx[4 ks + cq - x(n)]
  // (no centre), x(n) = n / 2 + 4 (n % 2) relative to the half
  double wyA[4], wxB[4];
  {
    const int xn = (r >> 1) + 4 * (r & 1);
#pragma unroll
    for (int ks = 0; ks < 4; ++ks) {
      const int d = 4 * ks + cq - r;
      wyA[ks] = (d >= 0 && d <= 8) ? (d == 4 ? p.wx[4] : p.wy[d]) : 0.0;
      const int e = 4 * ks + cq - xn;
      wxB[ks] = (e >= 0 && e <= 8 && e != 4) ? p.wx[e] : 0.0;
    }
  }
  // byte offsets in a stage: y arm operand (row 4 ks + cq, cell x(r) of the
  // half), x arm operand (row HAL + r, cells 8 hh + 4 ks + cq: the swizzle
  // exchanges even and odd k steps on odd rows), the thread's two centres
  const int jb = js * LY::JP;
  const int xn_r = (r >> 1) + 4 * (r & 1);
  const int offY = jb + halo_piece(cq, HAL + 8 * hh + xn_r) * 16;
  const int rowX = jb + ((HAL + r) * HX + 8 * hh + (cq ^ ((HAL + r) & 3))) * 16;
  const int offXe = rowX + 64 * pr, offXo = rowX + 64 * (1 - pr);
  const int offC0 = jb + halo_piece(HAL + r, HAL + xa) * 16;
  const int offC1 = jb + halo_piece(HAL + r, HAL + xb) * 16;
  const int offV0 = v_slot(r, xa) * 8, offV1 = v_slot(r, xb) * 8;
  [[maybe_unused]] const int offP0 = int(LY::o_psi0) + js * LY::JP0 + tile_piece(r, xa) * 16;
  [[maybe_unused]] const int offP1 = int(LY::o_psi0) + js * LY::JP0 + tile_piece(r, xb) * 16;

  const double fscale = p.fld_scale_dev ? *p.fld_scale_dev : 1.0;
  const double fz = p.fld[2] * fscale * B.h[2];
  const double fx0 = fscale * p.fld[0] * B.h[0], fy0 = fscale * p.fld[1] * B.h[1];
  const double fxy0 = fx0 * double(cx0 + xa + B.lo[0]) + fy0 * double(cy0 + r + B.lo[1]);
  const double fxy1 = fxy0 + 4.0 * fx0;
  const bool has_field = fz != 0.0 || fx0 != 0.0 || fy0 != 0.0;
  const double are = p.a_re, aim = p.a_im;
  double2 *out = static_cast<double2 *>(p.out);
  const long long out_ld = p.out_ld;
  const int ocol = chunk * LY::NS + js;
  double se = 0.0, sn = 0.0, sd = 0.0;
  [[maybe_unused]] const double dw0 =
      OBS ? p.obs_pol[0] * B.h[0] * double(cx0 + xa + B.lo[0]) + p.obs_pol[1] * B.h[1] * double(cy0 + r + B.lo[1])
          : 0.0;
  [[maybe_unused]] const double dw1 = OBS ? dw0 + 4.0 * p.obs_pol[0] * B.h[0] : 0.0;

  int gz0, gz1;
  {
    const int2 ca = __ldg(p.col_z + (long long)(cy0 + r) * B.NX + cx0 + xa);
    const int2 cb = __ldg(p.col_z + (long long)(cy0 + r) * B.NX + cx0 + xb);
    gz0 = min(ca.x, cb.x);
    gz1 = max(ca.y, cb.y);
  }

  // running sums [re, im][slot], .x / .y the thread's two cells: the pair
  // the accumulator fragment of a DMMA holds
  double2 ac[2][9];
#pragma unroll
  for (int q = 0; q < 2; ++q)
#pragma unroll
    for (int s = 0; s < 9; ++s) ac[q][s] = make_double2(0.0, 0.0);

  auto plane = [&](auto Kc, int k) {
    constexpr int K = decltype(Kc)::value;
    constexpr int S4 = (4 + K) % 9;
    cp_async_wait<NBUF - 2>();
    __syncthreads();
    const unsigned char *st = stage(k);
    const int pz = zbeg + k;
    if (__any_sync(0xffffffffu, pz >= gz0 - HAL && pz <= gz1 + HAL)) {
      double2 yb[4], xa4[4];
#pragma unroll
      for (int ks = 0; ks < 4; ++ks) yb[ks] = *reinterpret_cast<const double2 *>(st + offY + ks * (4 * HX * 16));
      xa4[0] = *reinterpret_cast<const double2 *>(st + offXe);
      xa4[1] = *reinterpret_cast<const double2 *>(st + offXo);
      xa4[2] = *reinterpret_cast<const double2 *>(st + offXe + 128);
      xa4[3] = *reinterpret_cast<const double2 *>(st + offXo + 128);
      const double2 u0 = *reinterpret_cast<const double2 *>(st + offC0);
      const double2 u1 = *reinterpret_cast<const double2 *>(st + offC1);
      // in-plane star into the running sums of output plane pz (slot S4)
#pragma unroll
      for (int ks = 0; ks < 4; ++ks) {
        dmma(ac[0][S4].x, ac[0][S4].y, wyA[ks], yb[ks].x);
        dmma(ac[1][S4].x, ac[1][S4].y, wyA[ks], yb[ks].y);
      }
#pragma unroll
      for (int ks = 0; ks < 4; ++ks) {
        dmma(ac[0][S4].x, ac[0][S4].y, xa4[ks].x, wxB[ks]);
        dmma(ac[1][S4].x, ac[1][S4].y, xa4[ks].y, wxB[ks]);
      }
      // local potential (+ laser) on the centres
      const double *vs = reinterpret_cast<const double *>(st + LY::o_v);
      double v0 = *reinterpret_cast<const double *>(reinterpret_cast<const unsigned char *>(vs) + offV0);
      double v1 = *reinterpret_cast<const double *>(reinterpret_cast<const unsigned char *>(vs) + offV1);
      if (has_field) {
        const double vz = fz * double(pz + B.lo[2]);
        v0 += fxy0 + vz;
        v1 += fxy1 + vz;
      }
      ac[0][S4].x = fma(v0, u0.x, ac[0][S4].x);
      ac[1][S4].x = fma(v0, u0.y, ac[1][S4].x);
      ac[0][S4].y = fma(v1, u1.x, ac[0][S4].y);
      ac[1][S4].y = fma(v1, u1.y, ac[1][S4].y);
      // z arm: plane pz feeds output planes pz - 4 .. pz + 4
#pragma unroll
      for (int jz = 0; jz < 9; ++jz) {
        if (jz == 4) continue;
        const double w = p.wz[8 - jz];
        const int s = (jz + K) % 9;
        ac[0][s].x = fma(w, u0.x, ac[0][s].x);
        ac[1][s].x = fma(w, u0.y, ac[1][s].x);
        ac[0][s].y = fma(w, u1.x, ac[0][s].y);
        ac[1][s].y = fma(w, u1.y, ac[1][s].y);
      }
    }
    // outputs of plane zo = pz - 4 are complete (slot K)
    const int zo = pz - HAL;
    if (zo >= zs) {
      const int *rows = reinterpret_cast<const int *>(side(k) + LY::s_rows);
      const int row0 = rows[row_slot(r, xa)], row1 = rows[row_slot(r, xb)];
      double pe = 0.0, pn = 0.0, pd = 0.0;
      (void)pe;
      (void)pn;
      (void)pd;
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int row = i ? row1 : row0;
        const double2 h = i ? make_double2(ac[0][K].y, ac[1][K].y) : make_double2(ac[0][K].x, ac[1][K].x);
        if (!(row >= 0 && row < p.np)) continue;
        double2 val = h;
        if constexpr (X0) {
          const double2 x0 = *reinterpret_cast<const double2 *>(st + (i ? offP1 : offP0));
          if constexpr (HORNER) {
            val.x = x0.x + are * h.x - aim * h.y;
            val.y = x0.y + are * h.y + aim * h.x;
          }
          if constexpr (OBS) {
            const double n2 = x0.x * x0.x + x0.y * x0.y;
            pe += x0.x * h.x + x0.y * h.y;
            pn += n2;
            pd += n2 * (i ? dw1 : dw0);
          }
        }
        out[row * out_ld + ocol] = val;
      }
      ac[0][K] = make_double2(0.0, 0.0);
      ac[1][K] = make_double2(0.0, 0.0);
      if constexpr (OBS) {
        se += pe;
        sn += pn;
        sd += pd + pn * (p.obs_pol[2] * B.h[2] * double(zo + B.lo[2]));
      }
    } else {
#pragma unroll
      for (int q = 0; q < 2; ++q) ac[q][K] = make_double2(0.0, 0.0);
    }
    issue_data(k + NBUF - 1);
    issue_side(k + LY::SIDE_AHEAD);
    cp_async_commit();
  };

#pragma unroll 1
  for (int k = 0; k < nplanes; k += 9) {
    plane(std::integral_constant<int, 0>{}, k);
#define HPSI_MMA_PLANE(J) \
  if (k + J < nplanes) plane(std::integral_constant<int, J>{}, k + J);
    HPSI_MMA_PLANE(1)
    HPSI_MMA_PLANE(2)
    HPSI_MMA_PLANE(3)
    HPSI_MMA_PLANE(4)
    HPSI_MMA_PLANE(5)
    HPSI_MMA_PLANE(6)
    HPSI_MMA_PLANE(7)
    HPSI_MMA_PLANE(8)
#undef HPSI_MMA_PLANE
  }
  cp_async_wait<0>();

  if constexpr (OBS) {
    // per-state sums: the 32 threads of a warp (fixed butterfly), then the two
    // warps of the state with a compensated sum
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      se += __shfl_xor_sync(0xffffffffu, se, off);
      sn += __shfl_xor_sync(0xffffffffu, sn, off);
      sd += __shfl_xor_sync(0xffffffffu, sd, off);
    }
    __syncthreads();
    double *red = reinterpret_cast<double *>(smem);
    if (ln == 0) {
      red[warp * 3 + 0] = se;
      red[warp * 3 + 1] = sn;
      red[warp * 3 + 2] = sd;
    }
    __syncthreads();
    if (tid < LY::NS) {
      double *o = p.obs + ((long long)ih * p.obs_ld + chunk * LY::NS + tid) * 6;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        Kahan a = {0.0, 0.0};
        kadd(a, red[(2 * tid) * 3 + c]);
        kadd(a, red[(2 * tid + 1) * 3 + c]);
        o[2 * c] = a.s;
        o[2 * c + 1] = a.c;
      }
    }
  }
}

template <bool HORNER, bool OBS>
hpsi_status launch_mode(const PassArgs &a, cudaStream_t st) {
  using LY = Layout<HORNER || OBS>;
  auto kern = pass_mma_kernel<HORNER, OBS>;
  static std::once_flag once;
  static cudaError_t attr = cudaSuccess;
  std::call_once(once, [&] {
    attr = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(LY::bytes));
  });
  HPSI_TRY_CUDA(attr);
  const unsigned nblocks = unsigned(a.nitems) * unsigned(a.chunks);
  kern<<<nblocks, LY::NT, LY::bytes, st>>>(a);
  HPSI_CHECK_LAUNCH();
  return HPSI_OK;
}

}  // namespace mma

// FP64 pass with the in-plane arms on DMMA: 16 x 8 tiles, 8-state chunks.
hpsi_status launch_pass_mma(const PassArgs &a, cudaStream_t st) {
  if (a.nitems == 0) return HPSI_OK;
  if (a.rho_part) {
    set_error("launch_pass_mma: the fused density is not built for this pass");
    return HPSI_ERR_UNSUPPORTED;
  }
  const bool horner = a.mode == PASS_HORNER, obs = a.obs != nullptr;
  if (horner && obs) return mma::launch_mode<true, true>(a, st);
  if (horner) return mma::launch_mode<true, false>(a, st);
  if (obs) return mma::launch_mode<false, true>(a, st);
  return mma::launch_mode<false, false>(a, st);
}

}  // namespace hpsi
