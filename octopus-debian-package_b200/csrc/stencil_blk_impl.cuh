// Templates of the register-blocked stencil pass (kernels, layouts and
// per-shape launchers), shared by the translation units that instantiate
// the cell-block shapes (stencil_blk.cu and stencil_blk_shapes_*.cu), so that
// the shapes compile in parallel.
#pragma once

#include <cuda.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <type_traits>
#include "stencil.cuh"
#include "stencil_blk.cuh"

namespace hpsi {
namespace blk {


// Lanes of one cell chunk: 128 bytes (FP64 16 = 8 complex states, FP32 32).
template <typename T>
constexpr int blk_lanes() {
  return 128 / int(sizeof(T));
}

// Element a thread owns per cell: one real lane, or one complex state.
template <typename T, bool CPLX>
struct BlkElem;
template <>
struct BlkElem<double, false> {
  using E = double;
};
template <>
struct BlkElem<float, false> {
  using E = float;
};
template <>
struct BlkElem<double, true> {
  using E = double2;
};
template <>
struct BlkElem<float, true> {
  using E = float2;
};
template <typename E>
__device__ __forceinline__ E ezero() {
  if constexpr (sizeof(E) == 16)
    return make_double2(0.0, 0.0);
  else if constexpr (sizeof(E) == 8 && !std::is_same<E, double>::value)
    return make_float2(0.f, 0.f);
  else
    return E(0);
}
__device__ __forceinline__ double fmae(double w, double v, double a) { return fma(w, v, a); }
__device__ __forceinline__ float fmae(float w, float v, float a) { return fmaf(w, v, a); }
__device__ __forceinline__ double2 fmae(double w, double2 v, double2 a) {
  return make_double2(fma(w, v.x, a.x), fma(w, v.y, a.y));
}
__device__ __forceinline__ float2 fmae(float w, float2 v, float2 a) {
  return __ffma2_rn(make_float2(w, w), v, a);  // packed FP32 multiply-add (sm_100)
}

template <typename T, bool X0, int RX_, int RY_, bool CPLX_, int TY_ = 8, int CB_ = 128>
struct BlkLayout {
  static constexpr bool CPLX = CPLX_;
  static constexpr int SL = CB_ / int(sizeof(T)), RX = RX_, RY = RY_;
  static constexpr int LW = CPLX ? 2 : 1;  // reals per thread element
  static constexpr int SLE = SL / LW;      // thread elements per cell chunk
  static constexpr int TX = BLK_TILE_X, TY = TY_, HAL = 4;
  static constexpr int HX = TX + 2 * HAL, HY = TY + 2 * HAL;
  static constexpr int HC = HX * HY, IC = TX * TY;
  static constexpr int CELLB = SL * int(sizeof(T));  // bytes of one cell chunk
  static constexpr int PCS = CELLB / 16;             // 16-byte pieces per cell chunk
  static constexpr int EPP = 16 / int(sizeof(T));    // elements per piece
  static_assert(CELLB == 128 || CELLB == 64, "cell chunks of 64 or 128 bytes");
  static constexpr int NT = SLE * (TX / RX) * (TY / RY);
  static_assert(NT == 256 || NT == 512, "256 or 512 threads");
  // 16-byte copy rounds of a halo plane / an interior plane (the last round
  // may be partial)
  static constexpr int IROUNDS = (IC * PCS + NT - 1) / NT;
  static constexpr bool IPART = (IC * PCS) % NT != 0;
  // the 25-point star reads no cell of the four HAL x HAL corners of the halo
  // plane: the fill gathers the SC star cells only (rows of the top and
  // bottom halo over the tile's columns, full halo rows beside the tile)
  static constexpr int SC = 2 * HAL * TX + TY * HX;
  static constexpr int SROUNDS = (SC * PCS + NT - 1) / NT;
  static constexpr bool SPART = (SC * PCS) % NT != 0;
  // two CTAs per SM for 256-thread blocks (shared memory <= 113 KB each)
  static constexpr int CTAS = (NT == 256 && CB_ == 64) ? 2 : 1;
  static constexpr int NBUF = (X0 || CTAS == 2) ? 3 : 4;  // data stages
  // side slots: >= 2 NBUF - 1 (issued 2 NBUF - 2 planes ahead); a power of 2
  // unless shared memory is short
  static constexpr int NSIDE = CTAS == 2 ? 2 * NBUF - 1 : 8;
  static constexpr int SIDE_AHEAD = 2 * NBUF - 2;
  // data stage: halo plane, psi0 rows of the output plane, potential
  static constexpr size_t o_psi0 = size_t(HC) * CELLB;
  static constexpr size_t o_v = o_psi0 + (X0 ? size_t(IC) * CELLB : 0);
  static constexpr size_t STAGE = o_v + size_t(IC) * sizeof(double);
  // side slot: load map of the halo plane, rows of the output plane 4 below
  static constexpr size_t s_rows = size_t(HC) * sizeof(int);
  static constexpr size_t SIDEB = s_rows + size_t(IC) * sizeof(int);
  static constexpr size_t o_side = NBUF * STAGE;
  // TMA fill: one mbarrier per data stage after the side ring
  static constexpr size_t o_mbar = o_side + NSIDE * SIDEB;
  static constexpr size_t bytes = o_mbar;
  static constexpr size_t bytes_tma = o_mbar + NBUF * 8;
  // mbarrier hand-over: a full and an empty barrier per data stage
  static constexpr size_t bytes_mb = o_mbar + 2 * NBUF * 8;
  static_assert(bytes * CTAS <= 232448 - 2048, "shared memory per CTA");
  static_assert(bytes_mb * CTAS <= 232448, "shared memory per CTA (mbarrier hand-over)");
  static_assert(STAGE % 16 == 0 && SIDEB % 16 == 0, "16-byte copies");
  static constexpr int NMAPP = HC / 4, NROWP = IC / 4, NVP = IC / 2;  // 16-byte side/v pieces
  static_assert(NMAPP + NROWP <= NT && NVP <= NT, "one side piece per thread");
  static_assert(NSIDE >= 2 * NBUF - 1, "side slot lifetime");
};

template <typename T>
__device__ __forceinline__ T wsel_t(const double *d, const float *f, int k);
template <>
__device__ __forceinline__ double wsel_t<double>(const double *d, const float *, int k) {
  return d[k];
}
template <>
__device__ __forceinline__ float wsel_t<float>(const double *, const float *f, int k) {
  return f[k];
}

__device__ __forceinline__ void zero16(void *d) {
  *reinterpret_cast<float4 *>(d) = make_float4(0.f, 0.f, 0.f, 0.f);
}
// Halo-plane cell (row-major in the HX x HY plane) of star cell i: i < HAL TX
// top rows over the tile's columns, then TY full rows, then the bottom rows.
template <class LY>
__device__ __forceinline__ int star_cell(int i) {
  constexpr int TX = LY::TX, TY = LY::TY, HX = LY::HX, HAL = LY::HAL;
  if (i < HAL * TX) return (i / TX) * HX + HAL + i % TX;
  i -= HAL * TX;
  if (i < TY * HX) return (HAL + i / HX) * HX + i % HX;
  i -= TY * HX;
  return (HAL + TY + i / TX) * HX + HAL + i % TX;
}

// Halo-plane cell of copy round j of copy cell c (c < NT / PCS) of the fill.
// With 16 x 8 tiles and 64 copy cells per round the five rounds cover the 320
// star cells as blocks with two per-thread bases: round 0 the top HAL rows over
// the tile's columns (row c / 16), round 4 the bottom rows (the same cells 12
// rows lower), rounds 1-3 the eight rows beside and across the tile in three
// column blocks of eight (row 4 + c / 8, column c % 8 + 8 (j - 1)), so that
// every round's cell is a base plus a constant.  Other shapes (and the TMA
// fill, whose segments follow the star order) use the star order.
template <class LY, bool STAR_ORDER>
__device__ __forceinline__ int fill_cell(int c, int j) {
  constexpr int HX = LY::HX, HAL = LY::HAL, TX = LY::TX;
  if constexpr (!STAR_ORDER && TX == 16 && LY::TY == 8 && LY::NT / LY::PCS == 64) {
    if (j == 0 || j == 4) return (c >> 4) * HX + HAL + (c & 15) + (j == 4 ? 12 * HX : 0);
    return (HAL + (c >> 3)) * HX + (c & 7) + 8 * (j - 1);
  } else {
    return star_cell<LY>(c + j * (LY::NT / LY::PCS));
  }
}

// 16-byte cp.async that reads `bytes` (16 or 0) and zero-fills the rest
__device__ __forceinline__ void cp_async16_zfill(void *smem, const void *gmem, int bytes) {
  unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(bytes));
}

// TMA fill helpers (hand-written PTX).  The tensor map covers the input batch
// as [rows][2 ld] elements with a box of 8 rows x one 128-byte chunk; the
// column coordinate is a chunk start (a multiple of 128 bytes).
__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  const unsigned a = static_cast<unsigned>(__cvta_generic_to_shared(bar));
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(a), "r"(count));
}
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, unsigned bytes) {
  const unsigned a = static_cast<unsigned>(__cvta_generic_to_shared(bar));
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(a), "r"(bytes) : "memory");
}
// true once the phase of the given parity has completed
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
  const unsigned a = static_cast<unsigned>(__cvta_generic_to_shared(bar));
  unsigned ok;
  asm volatile(
      "{\n .reg .pred P;\n mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n selp.u32 %0, 1, 0, P;\n}\n"
      : "=r"(ok)
      : "r"(a), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void tma_load_rows(void *dst, const CUtensorMap *tm, int x, int y, uint64_t *bar) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  const unsigned b = static_cast<unsigned>(__cvta_generic_to_shared(bar));
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(d),
      "l"(reinterpret_cast<uint64_t>(tm)), "r"(x), "r"(y), "r"(b)
      : "memory");
}
// polls of a stage's mbarrier before the pass gives up (a TMA copy that never
// lands: the kernel records HPSI_ERR_TIMEOUT in p.err and finishes without
// waiting further)
constexpr unsigned TMA_WAIT_LIMIT = 1u << 22;

// mbarrier hand-over of the stages (hand-written PTX).  The arrive-on of a
// thread's cp.async copies fires once all of them have landed; .noinc: the
// barrier's expected count already includes it.
__device__ __forceinline__ void cp_async_arrive_noinc(uint64_t *bar) {
  const unsigned a = static_cast<unsigned>(__cvta_generic_to_shared(bar));
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];\n" ::"r"(a) : "memory");
}
// plain arrive (release: the thread's earlier shared stores are visible to a
// thread that observes the phase)
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  const unsigned a = static_cast<unsigned>(__cvta_generic_to_shared(bar));
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(a) : "memory");
}

// grid: nitems (16 x 8 tiles x z blocks) * chunks.
// Plane k of a CTA is halo plane zbeg + k: data stage k % NBUF, side slot
// k % NSIDE.  Iteration k computes plane k and issues the data of plane
// k + NBUF - 1 and the side data of plane k + 2 NBUF - 2 (one commit group).
// One work unit: item ih (16 x 8 tile, z block) and state chunk `chunk`.
//
// MB: the stages change hands through mbarriers instead of one
// __syncthreads per plane.  Full barrier of a stage (2 NT arrivals per
// phase): every thread's cp.async arrive-on plus its plain arrive (covering
// its plain shared stores) after issuing a plane.  Empty barrier (NT): a
// thread arrives when it is done with a plane; the refill of that plane's
// stage waits for it.  The arrive comes after the arithmetic and the wait
// after the next plane's arithmetic, so a warp may run one plane ahead of the
// slowest one.  Every wait is bounded (HPSI_ERR_TIMEOUT in p.err).
template <typename T, bool HORNER, bool OBS, bool RHO, int U, int RX_, int RY_, bool CPLX, int TY_, int CB_,
          bool TMA = false, bool MB = false, bool FLD = true>
__device__ __forceinline__ void blk_body(const PassArgs &p, const int ih, const int chunk, unsigned char *smem,
                                         const CUtensorMap *tm = nullptr) {
  constexpr bool X0 = HORNER || OBS;
  using LY = BlkLayout<T, X0, RX_, RY_, CPLX, TY_, CB_>;
  using E = typename BlkElem<T, CPLX>::E;
  constexpr int SLE = LY::SLE;
  constexpr int SL = LY::SL, RX = LY::RX, RY = LY::RY, TX = LY::TX, TY = LY::TY, HAL = LY::HAL;
  constexpr int HX = LY::HX, NBUF = LY::NBUF, NSIDE = LY::NSIDE, PCS = LY::PCS, EPP = LY::EPP;

  const CellBox &B = p.box;
  const int4 it = p.items[ih];
  const int cx0 = HAL + it.x * TX, cy0 = HAL + it.y * TY;
  const int zs = it.z, ze = it.w;
  const int zbeg = zs - HAL, nplanes = ze - zs + 2 * HAL;
  const long long planeN = (long long)B.NX * B.NY;
  const int tid = threadIdx.x;
  const int col = chunk * SL;

  auto stage = [&](int k) { return smem + size_t(k % NBUF) * LY::STAGE; };
  auto side = [&](int k) { return smem + LY::o_side + size_t(k % NSIDE) * LY::SIDEB; };
  // TMA fill: star segment s (star cells 8 s .. 8 s + 7, eight consecutive
  // cells of one halo row) is one box copy when bit s of the plane's mask is
  // set (its rows are eight consecutive rows of the batch)
  static_assert(!TMA || (LY::TX == 16 && LY::TY == 8 && LY::CELLB == 128 && LY::SC == 320),
                "TMA fill: 16 x 8 tiles, 128-byte chunks");
  auto mbar = [&](int k) { return reinterpret_cast<uint64_t *>(smem + LY::o_mbar) + (k % NBUF); };
  [[maybe_unused]] const size_t mask_row = TMA ? (size_t(it.y) * p.seg_tiles_x + it.x) * B.NZ : 0;
  [[maybe_unused]] bool tma_dead = false;
  static_assert(!(TMA && MB), "one stage hand-over per kernel");
  // MB: full barrier of plane k's stage, empty barrier after it
  [[maybe_unused]] auto full_bar = [&](int k) { return reinterpret_cast<uint64_t *>(smem + LY::o_mbar) + (k % NBUF); };
  [[maybe_unused]] auto empty_bar = [&](int k) { return reinterpret_cast<uint64_t *>(smem + LY::o_mbar) + NBUF + (k % NBUF); };
  [[maybe_unused]] bool mb_dead = false;
  [[maybe_unused]] auto mb_wait = [&](uint64_t *bar, unsigned parity) {
    if (mb_dead) return;
    unsigned n = 0;
    while (!mbar_try_wait(bar, parity))
      if (++n == TMA_WAIT_LIMIT) {
        mb_dead = true;
        if (p.err) atomicExch(p.err, HPSI_ERR_TIMEOUT);
        return;
      }
  };
  [[maybe_unused]] const bool smem_a128 = (static_cast<unsigned>(__cvta_generic_to_shared(smem)) & 127u) == 0;

  // ---- copy roles ---------------------------------------------------------------
  const int cpc = tid / PCS, piece = tid % PCS;  // cell (+ NT / PCS per round) and 16-byte piece
  __builtin_assume(cpc >= 0 && cpc < LY::NT / PCS);
  const T *in_base = static_cast<const T *>(p.in) + col + piece * EPP;
  const long long in_ld2 = 2 * p.in_ld;
  const T *x0_base = static_cast<const T *>(p.psi0) + col + piece * EPP;
  // row strides in bytes (below 4 GiB, checked at launch): a row address is
  // one 32 x 32 -> 64-bit multiply-add of a non-negative row index
  const char *in_bytes = reinterpret_cast<const char *>(in_base);
  const unsigned in_rb = unsigned(in_ld2) * unsigned(sizeof(T));
  const char *x0_bytes = reinterpret_cast<const char *>(x0_base);
  const unsigned x0_rb = unsigned(2 * p.psi0_ld) * unsigned(sizeof(T));
  // side piece of this thread: map cells 4t..4t+3 (t < NMAPP), or rows cells
  long long side_src = 0;
  int side_dst = -1, side_kind = 0;  // 1 map, 2 rows
  if (tid < LY::NMAPP) {
    const int c = 4 * tid, hy = c / HX, hx = c % HX;
    side_kind = 1;
    side_dst = c;
    side_src = (long long)(cy0 - HAL + hy) * B.NX + cx0 - HAL + hx;
  } else if (tid < LY::NMAPP + LY::NROWP) {
    const int c = 4 * (tid - LY::NMAPP);
    side_kind = 2;
    side_dst = c;
    side_src = (long long)(cy0 + c / TX) * B.NX + cx0 + c % TX;
  }
  const int vc = 2 * tid;  // potential cells of this thread (tid < NVP)
  const long long v_src = (long long)(cy0 + vc / TX) * B.NX + cx0 + vc % TX;

  // side data of plane k (map of plane zbeg+k, rows of plane zbeg+k-4)
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
  // data of plane k: halo through the map, psi0 of the output plane, potential
  auto issue_data = [&](int k) {
    if (k >= nplanes) return;
    unsigned char *st = stage(k);
    const unsigned char *sd = side(k);
    const int *map = reinterpret_cast<const int *>(sd);
    T *halo = reinterpret_cast<T *>(st) + piece * EPP;
    [[maybe_unused]] unsigned long long mask = 0;
    if constexpr (TMA) {
      if (p.phase_corr == nullptr && smem_a128) mask = __ldg(p.seg_mask + mask_row + (zbeg + k));
      // the stage's mbarrier expects the bytes of every box of the plane (its
      // phase completes at once when the plane has none)
      if (tid == 0) mbar_arrive_expect_tx(mbar(k), unsigned(__popcll(mask)) * 8u * LY::CELLB);
    }
    if (p.phase_corr == nullptr) {
      // every entry is a row or -1 (zero): one zero-filling copy per piece
#pragma unroll
      for (int j = 0; j < LY::SROUNDS; ++j) {
        const int i = cpc + j * (LY::NT / PCS);
        if (LY::SPART && j == LY::SROUNDS - 1 && i >= LY::SC) break;
        if constexpr (TMA)
          if ((mask >> (i >> 3)) & 1ull) continue;  // this cell arrives with its segment's box
        const int cell = fill_cell<LY, TMA>(cpc, j);
        const int src = map[cell];
        cp_async16_zfill(halo + cell * SL, in_bytes + size_t(unsigned(max(src, 0))) * in_rb, src >= 0 ? 16 : 0);
      }
      if constexpr (TMA) {
        // thread s < 40 copies segment s
        if (tid < 40 && ((mask >> tid) & 1ull)) {
          // (the mask is cleared above when the dynamic shared memory is not
          // 128-byte aligned: box copies need 128-byte aligned destinations)
          const int cell = star_cell<LY>(8 * tid);
          tma_load_rows(reinterpret_cast<T *>(st) + cell * SL, tm, col, map[cell], mbar(k));
        }
      }
    } else {
#pragma unroll 1
      for (int j = 0; j < LY::SROUNDS; ++j) {
        const int i = cpc + j * (LY::NT / PCS);
        if (LY::SPART && j == LY::SROUNDS - 1 && i >= LY::SC) break;
        const int cell = star_cell<LY>(i);
        const int src = map[cell];
        T *d = halo + cell * SL;
        if (src >= 0) {
          cp_async16(d, in_base + src * in_ld2);
        } else if (src == -1) {
          zero16(d);
        } else {
          // periodic image times the Bloch phase correction
          const int b = -(src + 2);
          const T *g = in_base + __ldg(p.per_inner + b) * in_ld2;
          const T pr = static_cast<const T *>(p.phase_corr)[2 * b];
          const T pi = static_cast<const T *>(p.phase_corr)[2 * b + 1];
#pragma unroll
          for (int e = 0; e < EPP; e += 2) {
            const T xr = g[e], xi = g[e + 1];
            d[e] = xr * pr - xi * pi;
            d[e + 1] = xr * pi + xi * pr;
          }
        }
      }
    }
    const int q = zbeg + k;
    if (X0 && q - HAL >= zs) {
      const int *rows = reinterpret_cast<const int *>(sd + LY::s_rows);
      T *x0 = reinterpret_cast<T *>(st + LY::o_psi0) + piece * EPP;
#pragma unroll
      for (int j = 0; j < LY::IROUNDS; ++j) {
        const int cell = cpc + j * (LY::NT / PCS);
        if (LY::IPART && j == LY::IROUNDS - 1 && cell >= LY::IC) break;
        const int row = rows[cell];
        const bool ok = unsigned(row) < unsigned(p.np);  // row >= 0 && row < np
        cp_async16_zfill(x0 + cell * SL, x0_bytes + size_t(unsigned(ok ? row : 0)) * x0_rb, ok ? 16 : 0);
      }
    }
    if (tid < LY::NVP) {
      double *vd = reinterpret_cast<double *>(st + LY::o_v) + vc;
      if (p.v_cell)
        cp_async16(vd, p.v_cell + q * planeN + v_src);
      else
        zero16(vd);
    }
  };

  // ---- prologue: side data of planes 0..NBUF-2 synchronously, then the first
  // NBUF-1 groups (data of planes 0..NBUF-2, side of planes NBUF-1..2NBUF-3)
  if constexpr (TMA) {
    if (tid == 0) {
      for (int b = 0; b < NBUF; ++b) mbar_init(mbar(b), 1);
      mbar_init_fence();
    }
  }
  if constexpr (MB) {
    if (tid == 0) {
      for (int b = 0; b < NBUF; ++b) {
        mbar_init(full_bar(b), 2 * LY::NT);
        mbar_init(empty_bar(b), LY::NT);
      }
      mbar_init_fence();
    }
  }
  for (int k = 0; k < NBUF - 1 && k < nplanes; ++k) {
    unsigned char *sd = side(k);
    const int q = zbeg + k;
    for (int i = tid; i < LY::HC; i += LY::NT) {
      const int hy = i / HX, hx = i % HX;
      reinterpret_cast<int *>(sd)[i] = __ldg(p.cell_src + q * planeN + (long long)(cy0 - HAL + hy) * B.NX + cx0 - HAL + hx);
    }
    for (int i = tid; i < LY::IC; i += LY::NT)
      reinterpret_cast<int *>(sd + LY::s_rows)[i] =
          q - HAL >= zs ? __ldg(p.cell_row + (q - HAL) * planeN + (long long)(cy0 + i / TX) * B.NX + cx0 + i % TX)
                        : -1;
  }
  __syncthreads();
  for (int k = 0; k < NBUF - 1; ++k) {
    issue_data(k);
    issue_side(k + NBUF - 1);
    if constexpr (MB) {
      if (k < nplanes) {
        cp_async_arrive_noinc(full_bar(k));
        mbar_arrive(full_bar(k));
      }
    } else {
      cp_async_commit();
    }
  }

  // ---- compute roles --------------------------------------------------------------
  const int lane = tid & 31;
  const int l = tid % SLE;
  const int g = tid / SLE;
  const int bx = (g % (TX / RX)) * RX, by = (g / (TX / RX)) * RY;
  const double fscale = p.fld_scale_dev ? *p.fld_scale_dev : 1.0;
  const double fz = p.fld[2] * fscale * B.h[2];
  const double fx0 = fscale * p.fld[0] * B.h[0], fy0 = fscale * p.fld[1] * B.h[1];
  const double fxy0 = fx0 * double(cx0 + bx + B.lo[0]) + fy0 * double(cy0 + by + B.lo[1]);
  // uniform over the grid; FLD = false: compiled without the field term
  const bool has_field = FLD && (fz != 0.0 || fx0 != 0.0 || fy0 != 0.0);
  const T are = static_cast<T>(p.a_re), aim = static_cast<T>(p.a_im);
  const bool odd = !CPLX && (l & 1) != 0;
  // density weight of this lane's state (fused density of the output)
  [[maybe_unused]] const double wrho = RHO ? p.rho_w[col / 2 + (CPLX ? l : l / 2)] : 0.0;
  E *out = static_cast<E *>(p.out);
  const int ocol = col / LY::LW + l;
  char *out_bytes = reinterpret_cast<char *>(out + ocol);
  const unsigned out_rb = unsigned(2 * p.out_ld) * unsigned(sizeof(T));  // bytes per output row
  // observables: plain per-thread sums over the thread's z march (a few
  // hundred terms); the sums over threads and CTAs are compensated.  The x/y
  // part of the dipole weight of the thread's first cell, dxy00, is the only
  // per-cell constant kept live: fewer registers than per-cell norm sums
  double se = 0.0, sn = 0.0, sd = 0.0;
  const double dxy00 = OBS ? p.obs_pol[0] * B.h[0] * double(cx0 + bx + B.lo[0]) +
                                 p.obs_pol[1] * B.h[1] * double(cy0 + by + B.lo[1])
                           : 0.0;
  (void)se;
  (void)sn;
  (void)sd;
  (void)dxy00;
  (void)lane;

  // z range of the inner points under this thread's cells: planes more than
  // 4 away from it feed no output of the block and are skipped
  int gz0 = 1 << 30, gz1 = -(1 << 30);
#pragma unroll
  for (int r = 0; r < RY; ++r)
#pragma unroll
    for (int cx = 0; cx < RX; ++cx) {
      const int2 cz = __ldg(p.col_z + (long long)(cy0 + by + r) * B.NX + cx0 + bx + cx);
      gz0 = min(gz0, cz.x);
      gz1 = max(gz1, cz.y);
    }

  E acc[RX][RY][9];
#pragma unroll
  for (int cx = 0; cx < RX; ++cx)
#pragma unroll
    for (int r = 0; r < RY; ++r)
#pragma unroll
      for (int j = 0; j < 9; ++j) acc[cx][r][j] = ezero<E>();

  // one plane.  The running sums of a group of U planes sit in static slots:
  // plane K of the group adds its centre to slot (4 + K) % 9 and emits slot K;
  // after the group the nine slots rotate by U (U = 9 would need no rotation
  // but unrolls nine planes of code, more than the instruction cache holds).
  auto plane = [&](auto Kc, int k) {
    constexpr int K = decltype(Kc)::value;
    constexpr int S4 = (4 + K) % 9;  // running sum of output plane zbeg + k
    if constexpr (MB) {
      // the plane's copies and stores of every thread (and the side data of
      // plane k + NBUF - 1, issued with them)
      mb_wait(full_bar(k), unsigned(k / NBUF) & 1u);
    } else {
      cp_async_wait<NBUF - 2>();
      __syncthreads();
    }
    if constexpr (TMA) {
      // the plane's boxes (each thread observes the phase itself)
      if (!tma_dead) {
        unsigned n = 0;
        while (!mbar_try_wait(mbar(k), unsigned(k / NBUF) & 1u))
          if (++n == TMA_WAIT_LIMIT) {
            tma_dead = true;
            if (tid == 0 && p.err) atomicExch(p.err, HPSI_ERR_TIMEOUT);
            break;
          }
      }
    }
    // the refill of the stage read in plane k - 1 is issued after this
    // plane's arithmetic (every thread passed the barrier above, so the stage
    // is free): the arithmetic starts right after the barrier

    const unsigned char *st = stage(k);
    const E *P = reinterpret_cast<const E *>(st) + l;
    const double *vs = reinterpret_cast<const double *>(st + LY::o_v);
    const int pz = zbeg + k;
    const double vz = fz * double(pz + B.lo[2]);

    // warp-uniform test: a plane no cell of the warp needs is skipped by the
    // whole warp (its contributions would only reach non-inner outputs)
    if (__any_sync(0xffffffffu, pz >= gz0 - HAL && pz <= gz1 + HAL)) {
      // rows of the owned columns: y arms of every owned cell; the owned
      // cells themselves carry the centre (+ potential), the z arms and the x
      // arms of their siblings.  Columns innermost: consecutive multiply-adds
      // go to different running sums.
#pragma unroll
      for (int i = 0; i < RY + 8; ++i) {
#pragma unroll
        for (int cx = 0; cx < RX; ++cx) {
          const E val = P[((by + i) * HX + bx + cx + HAL) * SLE];
#pragma unroll
          for (int r = 0; r < RY; ++r) {
            const int d = i - r;
            if (d < 0 || d > 8) continue;
            if (d != 4) {
              acc[cx][r][S4] = fmae(wsel_t<T>(p.wy, p.wyf, d), val, acc[cx][r][S4]);
              continue;
            }
            double vv = vs[(by + r) * TX + bx + cx];
            if (has_field) vv += fxy0 + fx0 * double(cx) + fy0 * double(r) + vz;
            acc[cx][r][S4] = fmae(wsel_t<T>(p.wx, p.wxf, 4) + static_cast<T>(vv), val, acc[cx][r][S4]);
#pragma unroll
            for (int c2 = 0; c2 < RX; ++c2)
              if (c2 != cx) acc[c2][r][S4] = fmae(wsel_t<T>(p.wx, p.wxf, cx - c2 + 4), val, acc[c2][r][S4]);
            // slot (K + 8) % 9 was emitted by the previous plane: this is the
            // first term of its next output plane (no reset after the emit)
#pragma unroll
            for (int j = 0; j < 9; ++j)
              if (j != 4)
                acc[cx][r][(j + K) % 9] = fmae(wsel_t<T>(p.wz, p.wzf, 8 - j), val,
                                               j == 8 ? ezero<E>() : acc[cx][r][(j + K) % 9]);
          }
        }
      }
      // x arms from outside the owned block (rows innermost)
#pragma unroll
      for (int dx = -4; dx < RX + 4; ++dx) {
        if (dx >= 0 && dx < RX) continue;
#pragma unroll
        for (int r = 0; r < RY; ++r) {
          const E val = P[((by + r + HAL) * HX + bx + dx + HAL) * SLE];
#pragma unroll
          for (int cx = 0; cx < RX; ++cx) {
            const int dd = dx - cx;
            if (dd < -4 || dd > 4) continue;
            acc[cx][r][S4] = fmae(wsel_t<T>(p.wx, p.wxf, dd + 4), val, acc[cx][r][S4]);
          }
        }
      }
    } else {
      // skipped plane: the slot emitted by the previous plane starts at zero
#pragma unroll
      for (int cx = 0; cx < RX; ++cx)
#pragma unroll
        for (int r = 0; r < RY; ++r) acc[cx][r][(K + 8) % 9] = ezero<E>();
    }

    // outputs of plane zo = pz - 4 are complete (slot K)
    const int zo = pz - HAL;
    if (zo >= zs) {
      const int *rows = reinterpret_cast<const int *>(side(k) + LY::s_rows);
      [[maybe_unused]] const E *x0s = reinterpret_cast<const E *>(st + LY::o_psi0) + l;
      // output rows of the owned cells (pairs of x-adjacent cells in one load)
      int rowv[RX][RY];
#pragma unroll
      for (int r = 0; r < RY; ++r) {
        if constexpr (RX % 2 == 0) {
#pragma unroll
          for (int cx = 0; cx < RX; cx += 2) {
            const int2 rr = *reinterpret_cast<const int2 *>(rows + (by + r) * TX + bx + cx);
            rowv[cx][r] = rr.x;
            rowv[cx + 1][r] = rr.y;
          }
        } else {
#pragma unroll
          for (int cx = 0; cx < RX; ++cx) rowv[cx][r] = rows[(by + r) * TX + bx + cx];
        }
      }
      double pe = 0.0, pn = 0.0, pd = 0.0;
      (void)pe;
      (void)pn;
      (void)pd;
      [[maybe_unused]] double rc[RX * RY];
#pragma unroll
      for (int cx = 0; cx < RX; ++cx)
#pragma unroll
        for (int r = 0; r < RY; ++r) {
          [[maybe_unused]] const int cell = (by + r) * TX + bx + cx;
          const E h = acc[cx][r][K];
          E val = h;
          if constexpr (HORNER) {
            const E x0 = x0s[cell * SLE];
            if constexpr (CPLX) {
              val.x = x0.x + are * h.x - aim * h.y;
              val.y = x0.y + are * h.y + aim * h.x;
            } else {
              const T hp = __shfl_xor_sync(0xffffffffu, h, 1);  // the other part of this state
              val = odd ? x0 + are * h + aim * hp : x0 + are * h - aim * hp;
            }
          }
          const int row = rowv[cx][r];
          const bool ok = unsigned(row) < unsigned(p.np);  // row >= 0 && row < np
          if constexpr (RHO) {
            // this lane's share of the output's density, w_i |val_i|^2
            if constexpr (CPLX)
              rc[cx * RY + r] = ok ? wrho * (double(val.x) * double(val.x) + double(val.y) * double(val.y)) : 0.0;
            else
              rc[cx * RY + r] = ok ? wrho * double(val) * double(val) : 0.0;
          }
          if (!ok) continue;
          if constexpr (OBS) {
            const E x0 = x0s[cell * SLE];
            double eh, n2;
            if constexpr (CPLX) {
              eh = double(x0.x) * double(h.x) + double(x0.y) * double(h.y);
              n2 = double(x0.x) * double(x0.x) + double(x0.y) * double(x0.y);
            } else {
              eh = double(x0) * double(h);
              n2 = double(x0) * double(x0);
            }
            pe += eh;
            pn += n2;
            if (cx || r) pd += n2 * (double(cx) * (p.obs_pol[0] * B.h[0]) + double(r) * (p.obs_pol[1] * B.h[1]));
          }
          *reinterpret_cast<E *>(out_bytes + size_t(unsigned(row)) * out_rb) = val;
        }
      if constexpr (RHO) {
        // sum the NC = RX RY cell shares over the SLE lanes of the chunk: a
        // transposing butterfly halves the values a lane holds at each of the
        // first log2(NC) steps (one shuffle per kept pair), then a plain
        // reduction over the remaining lanes; lane l ends with the total of
        // cell sum_s hi_s NC / 2^(s+1).  5 double shuffles for 4 cells instead
        // of 16 (the shuffles share the MIO pipe with the stencil's loads).
        constexpr int NC = RX * RY;
        static_assert((NC & (NC - 1)) == 0 && NC <= SLE, "cells per thread: a power of 2 up to the lane group");
        int cell = 0;
#pragma unroll
        for (int st = 0; (NC >> st) > 1; ++st) {
          const int half = (NC >> st) / 2, off = SLE >> (st + 1);
          const bool hi = (l & off) != 0;
#pragma unroll
          for (int j = 0; j < half; ++j) {
            const double send = hi ? rc[j] : rc[j + half];
            const double keep = hi ? rc[j + half] : rc[j];
            rc[j] = keep + __shfl_xor_sync(0xffffffffu, send, off);
          }
          if (hi) cell += half;
        }
        constexpr int LOGNC = NC >= 8 ? 3 : NC >= 4 ? 2 : NC >= 2 ? 1 : 0;
#pragma unroll
        for (int off = SLE >> (LOGNC + 1); off > 0; off >>= 1) rc[0] += __shfl_xor_sync(0xffffffffu, rc[0], off);
        if ((l & ((SLE >> LOGNC) - 1)) == 0) {
          const int row = rowv[cell / RY][cell % RY];
          if (row >= 0 && row < p.np) p.rho_part[(long long)chunk * p.np + row] = rc[0];
        }
      }
      if constexpr (OBS) {
        // the plane's cells summed first, then one add per plane and sum;
        // dipole weight of a cell = dxy00 + its x/y offset terms (in pd) + z term
        se += pe;
        sn += pn;
        sd += pn * (dxy00 + p.obs_pol[2] * B.h[2] * double(zo + B.lo[2])) + pd;
      }
    }
    if constexpr (MB) {
      mbar_arrive(empty_bar(k));  // this thread is done with plane k
      const int kn = k + NBUF - 1;
      if (kn < nplanes) {
        // stage of plane k - 1 and the side slot of plane k + 2 NBUF - 2
        // (last held plane k - 1 or earlier): every thread done with k - 1
        if (k >= 1) mb_wait(empty_bar(k - 1), unsigned((k - 1) / NBUF) & 1u);
        issue_data(kn);
        issue_side(k + LY::SIDE_AHEAD);
        cp_async_arrive_noinc(full_bar(kn));
        mbar_arrive(full_bar(kn));
      }
    } else {
      issue_data(k + NBUF - 1);
      issue_side(k + LY::SIDE_AHEAD);
      cp_async_commit();
    }
  };

  auto rotate = [&]() {
#pragma unroll
    for (int cx = 0; cx < RX; ++cx)
#pragma unroll
      for (int r = 0; r < RY; ++r) {
        E t[9];
#pragma unroll
        for (int j = 0; j < 9; ++j) t[j] = acc[cx][r][(j + U) % 9];
#pragma unroll
        for (int j = 0; j < 9; ++j) acc[cx][r][j] = t[j];
      }
  };

#pragma unroll 1
  for (int k = 0; k < nplanes; k += U) {
    plane(std::integral_constant<int, 0>{}, k);
#define HPSI_BLK_PLANE(J)                                                          \
  if constexpr (U > J)                                                             \
    if (k + J < nplanes) plane(std::integral_constant<int, (U > J ? J : 0)>{}, k + J);
    HPSI_BLK_PLANE(1)
    HPSI_BLK_PLANE(2)
    HPSI_BLK_PLANE(3)
    HPSI_BLK_PLANE(4)
    HPSI_BLK_PLANE(5)
    HPSI_BLK_PLANE(6)
    HPSI_BLK_PLANE(7)
    HPSI_BLK_PLANE(8)
#undef HPSI_BLK_PLANE
    if constexpr (U % 9 != 0) rotate();
  }
  static_assert(U == 1 || U == 3 || U == 9, "groups of 1, 3 or 9 planes");
  cp_async_wait<0>();

  if constexpr (OBS) {
    // per-state sums over the threads of this chunk; the two lanes of a state
    // fold into one entry
    __syncthreads();
    double *red = reinterpret_cast<double *>(smem);  // threads x 6
    {
      double *o = red + tid * 6;
      o[0] = se;
      o[1] = 0.0;
      o[2] = sn;
      o[3] = 0.0;
      o[4] = sd;
      o[5] = 0.0;
    }
    __syncthreads();
    if (tid < SL / 2) {
      // threads of state tid: lanes 2 tid, 2 tid + 1 (real lanes) or lane tid
      Kahan a[3] = {{0, 0}, {0, 0}, {0, 0}};
      for (int t = LY::LW == 1 ? 2 * tid : tid; t < LY::NT; t += SLE)
        for (int q = 0; q < 3 - LY::LW; ++q)
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            kadd(a[c], red[(t + q) * 6 + 2 * c]);
            a[c].c += red[(t + q) * 6 + 2 * c + 1];
          }
      double *o = p.obs + ((long long)ih * p.obs_ld + chunk * (SL / 2) + tid) * 6;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        o[2 * c] = a[c].s;
        o[2 * c + 1] = a[c].c;
      }
    }
  }
}

template <typename T, bool HORNER, bool OBS, bool RHO, int U, int RX, int RY, bool CPLX, int TY, int CB, bool TMA,
          bool MB, bool FLD>
__global__ void __launch_bounds__(BlkLayout<T, HORNER || OBS, RX, RY, CPLX, TY, CB>::NT,
                                  BlkLayout<T, HORNER || OBS, RX, RY, CPLX, TY, CB>::CTAS)
    pass_blk_kernel(const __grid_constant__ PassArgs p, const __grid_constant__ CUtensorMap tm) {
  extern __shared__ __align__(128) unsigned char smem[];
  blk_body<T, HORNER, OBS, RHO, U, RX, RY, CPLX, TY, CB, TMA, MB, FLD>(p, blockIdx.x / p.chunks,
                                                                        blockIdx.x % p.chunks, smem, &tm);
}

// Many systems in one persistent launch (Horner passes): each CTA takes
// (system, item, chunk) units from a list sorted by cost until it is empty.
// FLD = false: no system of the launch has a laser field.
template <typename T, int U, int RX, int RY, bool CPLX, int TY, int CB, bool FLD>
__global__ void __launch_bounds__(BlkLayout<T, true, RX, RY, CPLX, TY, CB>::NT,
                                  BlkLayout<T, true, RX, RY, CPLX, TY, CB>::CTAS)
    pass_blk_group_kernel(const __grid_constant__ GroupArgs g) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ int unit_s;
  for (;;) {
    if (threadIdx.x == 0) unit_s = atomicAdd(g.counter, 1);
    __syncthreads();
    const int u = unit_s;
    __syncthreads();
    if (u >= g.nunits) break;
    const int4 W = g.units[u];  // {system, item, chunk, -}
    blk_body<T, true, false, false, U, RX, RY, CPLX, TY, CB, false, false, FLD>(g.sys[W.x], W.y, W.z, smem);
    __syncthreads();
  }
}

// The pass forms row addresses from 32-bit byte strides: every batch row
// (input, psi0, output) must be shorter than 4 GiB.
template <typename T>
bool blk_strides_ok(const PassArgs &a) {
  const long long lim = 0xffffffffll / (2 * (long long)sizeof(T));
  if (a.in_ld > lim || a.out_ld > lim || (a.psi0 && a.psi0_ld > lim)) {
    set_error("launch_pass_blk: a batch row is 4 GiB or longer");
    return false;
  }
  return true;
}

template <typename T, bool HORNER, bool OBS, bool RHO, int U, int RX, int RY, bool CPLX, int TY, int CB, bool TMA,
          bool MB, bool FLD>
hpsi_status launch_blk_mode(const PassArgs &a, const CUtensorMap *tm, cudaStream_t st) {
  using LY = BlkLayout<T, HORNER || OBS, RX, RY, CPLX, TY, CB>;
  constexpr size_t SMEM = TMA ? LY::bytes_tma : MB ? LY::bytes_mb : LY::bytes;
  auto kern = pass_blk_kernel<T, HORNER, OBS, RHO, U, RX, RY, CPLX, TY, CB, TMA, MB, FLD>;
  static std::once_flag once;
  static cudaError_t attr = cudaSuccess;
  std::call_once(once, [&] {
    attr = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(SMEM));
    if (attr == cudaSuccess && LY::CTAS > 1)
      attr = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  });
  HPSI_TRY_CUDA(attr);
  if (TMA && (!tm || !a.seg_mask)) {
    set_error("launch_pass_blk: TMA fill without its tensor map or segment masks");
    return HPSI_ERR_ARG;
  }
  if (!blk_strides_ok<T>(a)) return HPSI_ERR_ARG;
  CUtensorMap none;
  std::memset(&none, 0, sizeof(none));
  const unsigned nblocks = unsigned(a.nitems) * unsigned(a.chunks);
  kern<<<nblocks, LY::NT, SMEM, st>>>(a, tm ? *tm : none);
  HPSI_CHECK_LAUNCH();
  return HPSI_OK;
}

template <typename T, int U, int RX, int RY, bool CPLX, int TY, int CB, bool TMA, bool MB, bool FLD>
hpsi_status launch_blk_modes(const PassArgs &a, const CUtensorMap *tm, cudaStream_t st) {
  const bool horner = a.mode == PASS_HORNER, obs = a.obs != nullptr, rho = a.rho_part != nullptr;
  if (horner && obs) return launch_blk_mode<T, true, true, false, U, RX, RY, CPLX, TY, CB, TMA, MB, FLD>(a, tm, st);
  if (horner && rho) return launch_blk_mode<T, true, false, true, U, RX, RY, CPLX, TY, CB, TMA, MB, FLD>(a, tm, st);
  if (horner) return launch_blk_mode<T, true, false, false, U, RX, RY, CPLX, TY, CB, TMA, MB, FLD>(a, tm, st);
  if (obs) return launch_blk_mode<T, false, true, false, U, RX, RY, CPLX, TY, CB, TMA, MB, FLD>(a, tm, st);
  return launch_blk_mode<T, false, false, false, U, RX, RY, CPLX, TY, CB, TMA, MB, FLD>(a, tm, st);
}

template <typename T, int U, int RX, int RY, bool CPLX, int TY, int CB, bool TMA = false, bool MB = false>
hpsi_status launch_blk_u(const PassArgs &a, const CUtensorMap *tm, cudaStream_t st) {
  const bool horner = a.mode == PASS_HORNER, obs = a.obs != nullptr, rho = a.rho_part != nullptr;
  if (rho && (!horner || obs)) {
    set_error("launch_pass_blk: the density is fused into Horner passes without observables only");
    return HPSI_ERR_UNSUPPORTED;
  }
  // the default 16 x 8 shapes also come without the laser term, for passes
  // with no field set (fewer registers and branches per plane)
  constexpr bool NOFLD = !TMA && !MB && U == 9 && RX == 2 && RY == 2 && TY == 8 && CB == 128;
  if constexpr (NOFLD)
    if (a.fld[0] == 0.0 && a.fld[1] == 0.0 && a.fld[2] == 0.0)
      return launch_blk_modes<T, U, RX, RY, CPLX, TY, CB, TMA, MB, false>(a, tm, st);
  return launch_blk_modes<T, U, RX, RY, CPLX, TY, CB, TMA, MB, true>(a, tm, st);
}

template <typename T, int U, int RX, int RY, bool CPLX, int TY, int CB, bool FLD>
hpsi_status launch_blk_group_f(const GroupArgs &g, int grid, cudaStream_t st) {
  using LY = BlkLayout<T, true, RX, RY, CPLX, TY, CB>;
  auto kern = pass_blk_group_kernel<T, U, RX, RY, CPLX, TY, CB, FLD>;
  static std::once_flag once;
  static cudaError_t attr = cudaSuccess;
  std::call_once(once, [&] {
    attr = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(LY::bytes));
  });
  HPSI_TRY_CUDA(attr);
  kern<<<grid, LY::NT, LY::bytes, st>>>(g);
  HPSI_CHECK_LAUNCH();
  return HPSI_OK;
}

template <typename T, int U, int RX, int RY, bool CPLX, int TY, int CB>
hpsi_status launch_blk_group_v(const GroupArgs &g, int grid, cudaStream_t st) {
  bool fld = false;
  for (int s = 0; s < GROUP_MAX && g.sys[s].in != nullptr; ++s) {
    if (!blk_strides_ok<T>(g.sys[s])) return HPSI_ERR_ARG;
    fld = fld || g.sys[s].fld[0] != 0.0 || g.sys[s].fld[1] != 0.0 || g.sys[s].fld[2] != 0.0;
  }
  return fld ? launch_blk_group_f<T, U, RX, RY, CPLX, TY, CB, true>(g, grid, st)
             : launch_blk_group_f<T, U, RX, RY, CPLX, TY, CB, false>(g, grid, st);
}

// chunk bytes of a shape: sc complex states of the storage type
template <typename T>
int shape_cb(const PassShape &s) {
  return s.sc * 2 * int(sizeof(T));
}


}  // namespace blk
}  // namespace hpsi
