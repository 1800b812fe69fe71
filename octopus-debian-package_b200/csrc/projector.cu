// Kleinman-Bylander projector "bra": projections of a batch on the projector
// spheres, the step X(hamiltonian_elec_base_nlocal_start) performs on the CPU
// as a gather of the sphere points followed by a real GEMM
// (src/hamiltonian/hamiltonian_elec_base_inc.F90:650-780):
//   proj[row0(m) + j][s] = scal[j] * sum_k P_m[k][j] * psi[map_m[k]][s].
// The matching "ket" (add P * proj back onto the covered rows) runs per
// covered row after the stencil pass: one thread per output element, so no
// write races and no colouring are needed.
//
// The contraction runs on the FP64 tensor cores (DMMA,
// mma.sync.m8n8k4.f64) for both storage types: M = 8 real lanes per warp,
// N = 8 projectors per tile, K = 4 sphere points per step, with the gathered
// rows and the projector block staged in shared memory by cp.async.  The SIMT
// kernel below serves matrices with more than 16 projectors and is the
// cross-check of the tensor path.
#include <algorithm>
#include <cstdlib>
#include <type_traits>

#include "projector.cuh"

namespace hpsi {

namespace {

constexpr int KB = 32;     // sphere points per staged block
constexpr int LANES = 32;  // real lanes per CTA (16 complex states)
constexpr int APAD = 40;   // padded row length of the staged psi block (doubles)
constexpr int NMAX = 16;   // projectors per matrix served by the DMMA kernel

// 8-byte cp.async that reads `bytes` (8 or 0) and zero-fills the rest
__device__ __forceinline__ void cp_async8_zfill(void *smem, const void *gmem, int bytes) {
  unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gmem), "r"(bytes));
}

__device__ __forceinline__ void dmma_m8n8k4(double &d0, double &d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// grid: (nmat, ld2 / LANES, ksplit); block: 128 threads (4 warps x 8 lanes
// each).  Split z sums sphere points [z*npts/ksplit, (z+1)*npts/ksplit) into
// partial[z] (unscaled, FP64); bra_reduce_kernel adds the splits and applies
// scal.  T is the storage type of psi: FP32 rows are staged as stored and
// widened to FP64 when the A fragment is read, so both precisions contract
// in FP64 against the FP64 projector values.
template <typename T>
__global__ void __launch_bounds__(128) bra_dmma_kernel(const ProjArgs p) {
  constexpr int AP = sizeof(T) == 8 ? APAD : 40;  // 40 floats: conflict-free fragment reads
  constexpr int CPR = LANES * int(sizeof(T)) / 16;  // 16-byte copies per staged row
  constexpr int NS = 3;  // staged blocks: two in flight while one is contracted
  __shared__ __align__(16) T sA[NS][KB][AP];
  __shared__ __align__(16) double sB[NS][KB][NMAX];
  const int m = blockIdx.x;
  const int l0 = blockIdx.y * LANES;
  const int4 md = p.mat[m];  // npoints, nproj, map_off, pt_off
  const int kbeg = int((long long)md.x * blockIdx.z / gridDim.z);
  const int kend = int((long long)md.x * (blockIdx.z + 1) / gridDim.z);
  const int npts = kend - kbeg, npr = md.y;
  const int *map = p.map + md.z + kbeg;
  const double *pt = p.pt64 + md.w + (long long)kbeg * npr;
  const T *psi = static_cast<const T *>(p.psi);
  const long long ld2 = 2 * p.psi_ld;
  const int tid = threadIdx.x, warp = tid >> 5, ln = tid & 31;
  constexpr int EPC = 16 / int(sizeof(T));  // elements per 16-byte copy

  // the map entries of the next staged block are loaded one block ahead into
  // registers, so a row copy never waits for its own index load
  constexpr int NIT = KB * CPR / 128;  // row pieces per thread and block
  static_assert(KB * CPR % 128 == 0, "whole rounds of row pieces");
  int mrow[NIT];
  auto load_map = [&](int k0) {
#pragma unroll
    for (int t = 0; t < NIT; ++t) {
      const int k = (tid + 128 * t) / CPR;
      mrow[t] = k0 + k < npts ? __ldg(map + k0 + k) : 0;
    }
  };
  auto stage = [&](int k0, int b) {
#pragma unroll
    for (int t = 0; t < NIT; ++t) {
      const int i = tid + 128 * t;
      const int k = i / CPR, part = i % CPR;
      T *d = &sA[b][k][part * EPC];
      if (k0 + k < npts && l0 + part * EPC < ld2) {
        cp_async16(d, psi + mrow[t] * ld2 + l0 + part * EPC);
      } else {
        *reinterpret_cast<float4 *>(d) = make_float4(0.f, 0.f, 0.f, 0.f);
      }
    }
    for (int i = tid; i < KB * NMAX; i += 128) {
      const int k = i / NMAX, j = i % NMAX;
      const bool ok = k0 + k < npts && j < npr;
      cp_async8_zfill(&sB[b][k][j], ok ? pt + (long long)(k0 + k) * npr + j : p.pt64, ok ? 8 : 0);
    }
  };

  double c0[2] = {0.0, 0.0}, c1[2] = {0.0, 0.0};
  const int nblk = (npts + KB - 1) / KB;
  load_map(0);
  if (nblk > 0) stage(0, 0);
  cp_async_commit();
  load_map(KB);
  if (nblk > 1) stage(KB, 1);
  cp_async_commit();
  load_map(2 * KB);
  for (int blk = 0; blk < nblk; ++blk) {
    const int b = blk % NS;
    if (blk + 2 < nblk) stage((blk + 2) * KB, (blk + 2) % NS);
    cp_async_commit();
    load_map((blk + 3) * KB);
    cp_async_wait<2>();
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < KB; kk += 4) {
      const double a = double(sA[b][kk + (ln & 3)][warp * 8 + (ln >> 2)]);
#pragma unroll
      for (int nt = 0; nt < 2; ++nt) {
        const double bb = sB[b][kk + (ln & 3)][nt * 8 + (ln >> 2)];
        dmma_m8n8k4(c0[nt], c1[nt], a, bb);
      }
    }
    __syncthreads();
  }
  cp_async_wait<0>();
  // C fragment: row (lane) = ln >> 2, cols (projectors) = (ln & 3) * 2 + {0,1}
  const int lane = l0 + warp * 8 + (ln >> 2);
  if (lane >= ld2) return;  // lanes past the batch width (zero-filled above)
  double *out = p.partial + ((long long)blockIdx.z * p.nprojections + p.proj_row[m]) * 2 * p.proj_ld;
#pragma unroll
  for (int nt = 0; nt < 2; ++nt) {
    const int j0 = nt * 8 + (ln & 3) * 2;
    if (j0 < npr) out[(long long)j0 * 2 * p.proj_ld + lane] = c0[nt];
    if (j0 + 1 < npr) out[(long long)(j0 + 1) * 2 * p.proj_ld + lane] = c1[nt];
  }
}

// proj[j][l] = scal[j] * sum_z partial[z][j][l]  (one thread per real lane;
// FP64 sums, rounded once to the storage type)
template <typename T>
__global__ void bra_reduce_kernel(const ProjArgs p, int ksplit) {
  const long long n = (long long)p.nprojections * 2 * p.proj_ld;
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int j = int(i / (2 * p.proj_ld));
  double acc = 0.0;
  for (int z = 0; z < ksplit; ++z) acc += p.partial[(long long)z * n + i];
  static_cast<T *>(p.proj)[i] = T(acc * p.scal64[j]);
}

// SIMT bra: grid (nmat, ceil(ld2/32)); block 128 = 32 lanes x 4 point groups.
// PHASE: each gathered point is first multiplied by its projector phase
// (lpsi = psi(map) * projector_phases, hamiltonian_elec_base_inc.F90:680-701);
// lane pairs (2s, 2s + 1) hold one complex number, exchanged by a shuffle.
template <typename T, bool PHASE>
__global__ void __launch_bounds__(128) bra_simt_kernel(const ProjArgs p) {
  constexpr int MAXP = 32;
  __shared__ T red[4][MAXP][32];
  const int m = blockIdx.x;
  const int ln = threadIdx.x & 31, grp = threadIdx.x >> 5;
  const long long ld2 = 2 * p.psi_ld;
  const int lane = blockIdx.y * 32 + ln;
  const int4 md = p.mat[m];
  const int npts = md.x, npr = md.y;
  const int *map = p.map + md.z;
  const T *pt = static_cast<const T *>(p.pt) + md.w;
  const T *psi = static_cast<const T *>(p.psi);
  T acc[MAXP];
#pragma unroll
  for (int j = 0; j < MAXP; ++j) acc[j] = T(0);
  if constexpr (!PHASE) {
    if (lane < ld2) {
      for (int k = grp; k < npts; k += 4) {
        const T x = psi[__ldg(map + k) * ld2 + lane];
        const T *pk = pt + (long long)k * npr;
#pragma unroll
        for (int j = 0; j < MAXP; ++j)
          if (j < npr) acc[j] += pk[j] * x;
      }
    }
  } else {
    // every lane of the warp runs the loop (the shuffle needs all 32)
    const T *ph = static_cast<const T *>(p.phase) + 2 * (long long)md.z;
    for (int k = grp; k < npts; k += 4) {
      T x = lane < ld2 ? psi[__ldg(map + k) * ld2 + lane] : T(0);
      const T other = __shfl_xor_sync(0xffffffffu, x, 1);
      const T c = ph[2 * k], sn = ph[2 * k + 1];
      x = (ln & 1) ? other * sn + x * c : x * c - other * sn;
      const T *pk = pt + (long long)k * npr;
#pragma unroll
      for (int j = 0; j < MAXP; ++j)
        if (j < npr) acc[j] += pk[j] * x;
    }
  }
#pragma unroll
  for (int j = 0; j < MAXP; ++j) red[grp][j][ln] = acc[j];
  __syncthreads();
  if (grp == 0 && lane < ld2) {
    const T *scal = static_cast<const T *>(p.scal) + p.proj_row[m];
    T *out = static_cast<T *>(p.proj) + (long long)p.proj_row[m] * 2 * p.proj_ld;
    for (int j = 0; j < npr; ++j) {
      const T s = red[0][j][ln] + red[1][j][ln] + red[2][j][ln] + red[3][j][ln];
      out[(long long)j * 2 * p.proj_ld + lane] = s * scal[j];
    }
  }
}

}  // namespace

int bra_ksplit(const ProjArgs &p, int num_sms) {
  const long long ld2 = 2 * p.psi_ld;
  const long long base = (long long)p.nmat * ((ld2 + LANES - 1) / LANES);
  static const long long target = [] {
    const char *e = std::getenv("HPSI_BRA_CTAS_PER_SM");  // tuning override
    return e ? std::max(1, std::atoi(e)) : 32;  // measured: 4 -> 0.196 ms, 16 -> 0.188, 32 -> 0.174 (R = 12 sphere)
  }();
  long long k = (target * num_sms + base - 1) / base;
  k = std::min<long long>(k, std::max(1, p.min_npoints / 128));
  return int(std::max<long long>(1, std::min<long long>(k, 64)));
}

template <typename T>
hpsi_status launch_bra(const ProjArgs &p, bool use_tensor, int ksplit, cudaStream_t st) {
  if (p.nmat == 0) return HPSI_OK;
  const long long ld2 = 2 * p.psi_ld;
  // the staged rows are copied in 16-byte pieces: FP32 needs an even width
  if (p.phase) {  // projector phases: the SIMT kernel rotates each gathered point
    if (p.max_nproj > 32) {
      set_error("projector matrices with more than 32 projectors are not supported");
      return HPSI_ERR_UNSUPPORTED;
    }
    dim3 grid(p.nmat, unsigned((ld2 + 31) / 32));
    bra_simt_kernel<T, true><<<grid, 128, 0, st>>>(p);
    HPSI_CHECK_LAUNCH();
    return HPSI_OK;
  }
  if (use_tensor && p.max_nproj <= NMAX && ld2 % (16 / sizeof(T)) == 0) {
    dim3 grid(p.nmat, unsigned((ld2 + LANES - 1) / LANES), ksplit);
    bra_dmma_kernel<T><<<grid, 128, 0, st>>>(p);
    HPSI_CHECK_LAUNCH();
    const long long n = (long long)p.nprojections * ld2;
    bra_reduce_kernel<T><<<unsigned((n + 255) / 256), 256, 0, st>>>(p, ksplit);
    HPSI_CHECK_LAUNCH();
    return HPSI_OK;
  }
  if (p.max_nproj > 32) {
    set_error("projector matrices with more than 32 projectors are not supported");
    return HPSI_ERR_UNSUPPORTED;
  }
  dim3 grid(p.nmat, unsigned((ld2 + 31) / 32));
  bra_simt_kernel<T, false><<<grid, 128, 0, st>>>(p);
  HPSI_CHECK_LAUNCH();
  return HPSI_OK;
}

// ---------------------------------------------------------------------------
// KB ket, one thread per (covered row, complex state): h = sum over the
// row's (matrix, point) entries of P[point][j] * proj[j], then
// out[row] += h (apply) or += a * h (Horner pass), and, if requested, the
// energy partial Re(conj(psi0[row]) h) per state.  Each output element is
// written by exactly one thread, in a fixed order: no atomics, deterministic.
namespace {
// RPW rows per warp: 1 for batches wider than 16 states; narrow batches (at
// most 16 or 8 states) put 2 or 4 rows in a warp, one lane group of 32 / RPW
// lanes per row, so the lanes past the batch width do not idle.
template <typename T, typename C2, bool PHASE, int RPW = 1>
__global__ void __launch_bounds__(256) ket_kernel(const KetArgs k) {
  // each thread serves two states (sb, sb + 32) of its rows: the row's
  // metadata and projector weights are loaded once for both (12 % faster than
  // one state per thread on the R = 12 sphere, 128 states; four states per
  // thread measured 30 % slower, the grid no longer filling the GPU)
  constexpr int L = 32 / RPW;            // lanes per row
  constexpr int SPT = RPW == 1 ? 2 : 1;  // states per thread
  const int lane = threadIdx.x % L, sub = threadIdx.x / L;
  const int sb = blockIdx.x * L * SPT + lane;
  bool act[SPT];
#pragma unroll
  for (int u = 0; u < SPT; ++u) act[u] = sb + L * u < k.nst;
  const T *pt = static_cast<const T *>(k.pt);
  const C2 *proj = static_cast<const C2 *>(k.proj);
  C2 *out = static_cast<C2 *>(k.out);
  const C2 *psi0 = static_cast<const C2 *>(k.psi0);
  Kahan ke[SPT];
#pragma unroll
  for (int u = 0; u < SPT; ++u) ke[u] = {0, 0};
  // each CTA row takes a contiguous range of covered rows: neighbouring rows
  // lie in the same few spheres, so their projections stay in L1
  const int per = (k.nk + gridDim.y - 1) / gridDim.y;
  const int r0 = blockIdx.y * per, r1 = min(k.nk, r0 + per);
  for (int i0 = r0 + threadIdx.y * RPW; i0 < r1; i0 += 8 * RPW) {
    // row of this lane group; density of the final row (the loop bound is
    // the same for the whole warp: the shuffle below is reached by all its
    // lanes, active or not)
    const int i = i0 + sub;
    const bool rv = i < r1;
    double rs = 0.0;
    if (act[0] && rv) {
    const int row = k.krows[i];
    // the output elements are loaded before the sums, so their latency
    // overlaps theirs (prefetching the next row's metadata as well, or four
    // rows per warp, measured slower)
    C2 *o = out + (long long)row * k.out_ld + sb;
    C2 y[SPT], h[SPT];
#pragma unroll
    for (int u = 0; u < SPT; ++u) {
      if (act[u]) y[u] = o[L * u];
      h[u].x = 0;
      h[u].y = 0;
    }
    for (int e = k.kptr[i]; e < k.kptr[i + 1]; ++e) {
      const int4 E = __ldg(k.ent + e);
      const T *pp = pt + E.x;
      const C2 *pr = proj + (long long)E.y * k.proj_ld + sb;
      if constexpr (!PHASE) {
        for (int j = 0; j < E.z; ++j) {
          const T w = pp[j];
#pragma unroll
          for (int u = 0; u < SPT; ++u) {
            if (!act[u]) continue;
            const C2 v = pr[(long long)j * k.proj_ld + L * u];
            h[u].x += w * v.x;
            h[u].y += w * v.y;
          }
        }
      } else {
        // this point's contribution times conj(phase) (the ket of
        // hamiltonian_elec_base_inc.F90:934-1025 with projector phases)
        C2 g[SPT];
#pragma unroll
        for (int u = 0; u < SPT; ++u) g[u].x = g[u].y = 0;
        for (int j = 0; j < E.z; ++j) {
          const T w = pp[j];
#pragma unroll
          for (int u = 0; u < SPT; ++u) {
            if (!act[u]) continue;
            const C2 v = pr[(long long)j * k.proj_ld + L * u];
            g[u].x += w * v.x;
            g[u].y += w * v.y;
          }
        }
        const T *ph = static_cast<const T *>(k.phase) + 2 * (long long)E.w;
        const T c = ph[0], sn = ph[1];
#pragma unroll
        for (int u = 0; u < SPT; ++u) {
          h[u].x += g[u].x * c + g[u].y * sn;
          h[u].y += g[u].y * c - g[u].x * sn;
        }
      }
    }
#pragma unroll
    for (int u = 0; u < SPT; ++u) {
      if (!act[u]) continue;
      if (k.mode == 1) {
        const T ar = T(k.a_re), ai = T(k.a_im);
        y[u].x += ar * h[u].x - ai * h[u].y;
        y[u].y += ar * h[u].y + ai * h[u].x;
      } else {
        y[u].x += h[u].x;
        y[u].y += h[u].y;
      }
      o[L * u] = y[u];
      if (k.rho_ket) rs += k.rho_w[sb + L * u] * (double(y[u].x) * double(y[u].x) + double(y[u].y) * double(y[u].y));
      if (k.obs) {
        const C2 x = psi0[(long long)row * k.psi0_ld + sb + L * u];
        kadd(ke[u], double(x.x) * double(h[u].x) + double(x.y) * double(h[u].y));
      }
    }
    }
    if (k.rho_ket) {
      // sum over the row's lane group (xor offsets below L stay inside it)
      for (int off = L / 2; off > 0; off >>= 1) rs += __shfl_xor_sync(0xffffffffu, rs, off);
      if (lane == 0 && rv) k.rho_ket[(long long)blockIdx.x * k.nk + i] = rs;
    }
  }
  if (k.obs) {
    __shared__ double red[8][32 * SPT][2];
#pragma unroll
    for (int u = 0; u < SPT; ++u) {
      red[threadIdx.y][threadIdx.x + 32 * u][0] = ke[u].s;
      red[threadIdx.y][threadIdx.x + 32 * u][1] = ke[u].c;
    }
    __syncthreads();
    if (threadIdx.y == 0 && sub == 0) {
#pragma unroll
      for (int u = 0; u < SPT; ++u) {
        if (!act[u]) continue;
        Kahan a = {0, 0};
        for (int y = 0; y < 8; ++y)
          for (int q = 0; q < RPW; ++q) {
            kadd(a, red[y][q * L + lane + 32 * u][0]);
            a.c += red[y][q * L + lane + 32 * u][1];
          }
        double *o = k.obs + ((long long)blockIdx.y * k.obs_ld + sb + L * u) * 2;
        o[0] = a.s;
        o[1] = a.c;
      }
    }
  }
}
}  // namespace

// At most 1024 CTA rows, each over a contiguous range of covered rows: one
// row per thread (up to 65535 CTA rows) measured 45 % slower on the R = 12
// sphere, the projections of neighbouring rows no longer sharing L1.
int ket_row_blocks(int nk) {
  static const int cap = [] {
    const char *e = std::getenv("HPSI_KET_ROW_BLOCKS");  // tuning override
    return e ? std::max(1, std::min(65535, std::atoi(e))) : 1024;
  }();
  return std::max(1, std::min(cap, (nk + 7) / 8));
}

template <typename T>
hpsi_status launch_ket(const KetArgs &k, cudaStream_t st) {
  if (k.nk == 0) return HPSI_OK;
  using C2 = typename std::conditional<sizeof(T) == 8, double2, float2>::type;
  const int rb = k.row_blocks > 0 ? std::min(k.row_blocks, ket_row_blocks(k.nk)) : ket_row_blocks(k.nk);
  dim3 grid((k.nst + 63) / 64, rb);  // two states per thread
  // narrow batches: several rows per warp
  const int rpw = k.nst <= 8 ? 4 : k.nst <= 16 ? 2 : 1;
  if (k.phase) {
    if (rpw == 4)
      ket_kernel<T, C2, true, 4><<<grid, dim3(32, 8), 0, st>>>(k);
    else if (rpw == 2)
      ket_kernel<T, C2, true, 2><<<grid, dim3(32, 8), 0, st>>>(k);
    else
      ket_kernel<T, C2, true><<<grid, dim3(32, 8), 0, st>>>(k);
  } else {
    if (rpw == 4)
      ket_kernel<T, C2, false, 4><<<grid, dim3(32, 8), 0, st>>>(k);
    else if (rpw == 2)
      ket_kernel<T, C2, false, 2><<<grid, dim3(32, 8), 0, st>>>(k);
    else
      ket_kernel<T, C2, false><<<grid, dim3(32, 8), 0, st>>>(k);
  }
  HPSI_CHECK_LAUNCH();
  return HPSI_OK;
}

template hpsi_status launch_ket<double>(const KetArgs &, cudaStream_t);
template hpsi_status launch_ket<float>(const KetArgs &, cudaStream_t);

template hpsi_status launch_bra<double>(const ProjArgs &, bool, int, cudaStream_t);
template hpsi_status launch_bra<float>(const ProjArgs &, bool, int, cudaStream_t);

}  // namespace hpsi
