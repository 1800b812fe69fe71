// Shared definitions of the hpsi CUDA library (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <string>

#include "../../include/hpsi.h"

namespace hpsi {

// ---------------------------------------------------------------------------
// error reporting
void set_error(const std::string &msg);
extern std::atomic<int64_t> g_launches;

#define HPSI_TRY_CUDA(expr)                                                    \
  do {                                                                         \
    cudaError_t e_ = (expr);                                                   \
    if (e_ != cudaSuccess) {                                                   \
      ::hpsi::set_error(std::string(#expr) + ": " + cudaGetErrorString(e_));   \
      return HPSI_ERR_CUDA;                                                    \
    }                                                                          \
  } while (0)

#define HPSI_CHECK_LAUNCH()                                                    \
  do {                                                                         \
    ::hpsi::g_launches.fetch_add(1, std::memory_order_relaxed);                \
    cudaError_t e_ = cudaGetLastError();                                       \
    if (e_ != cudaSuccess) {                                                   \
      ::hpsi::set_error(std::string("kernel launch: ") +                       \
                        cudaGetErrorString(e_));                               \
      return HPSI_ERR_CUDA;                                                    \
    }                                                                          \
  } while (0)

// ---------------------------------------------------------------------------
// cell box geometry shared by all kernels of one mesh
struct CellBox {
  int NX, NY, NZ;       // padded cell box (halo of `halo` cells on each side)
  int nxo, nyo, nzo;    // inner bounding box extent (outputs live here)
  int lo[3];            // integer coordinate of cell (0,0,0)
  int halo;             // = stencil order (4)
  double h[3];          // spacing
};

// ---------------------------------------------------------------------------
// compensated (two-sum) FP64 accumulation
struct Kahan {
  double s, c;
};
__host__ __device__ inline void kadd(Kahan &k, double x) {
  double t = k.s + x;
  double bp = t - k.s;
  double err = (k.s - (t - bp)) + (x - bp);
  k.s = t;
  k.c += err;
}
__host__ __device__ inline void kmerge(Kahan &a, const Kahan &b) {
  kadd(a, b.s);
  a.c += b.c;
}

// ---------------------------------------------------------------------------
// cp.async helpers (16-byte, L2-only caching for streamed data)
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem) {
  unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem) {
  unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::);
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

}  // namespace hpsi
