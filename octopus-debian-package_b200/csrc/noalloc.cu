// Allocation-free state norms.
//
// hpsi_nrm2 keeps its per-block partial sums in a workspace that the mesh
// handle allocates on first use.  Some callers cannot allocate device memory
// at the point where they need a norm: code running under a memory pool or a
// device-memory budget owned by someone else (a host application that
// forbids the library from calling cudaMalloc), or a tight per-step loop that
// must not hit the allocator.  This entry point takes only the sizes it needs
// and keeps its partial sums in one file-scope device array instead.
//
// The array below has a fixed maximum size; every GPU that loads the library
// holds it until the process exits.  Host code never dereferences or passes
// the symbol itself: its device address is looked up once per device with
// cudaGetSymbolAddress and that address is handed to the kernels.
#include <mutex>
#include <string>
#include <vector>

#include "api_internal.cuh"
#include "reduce.cuh"

namespace hpsi {

namespace {

constexpr int NOALLOC_BLOCKS = 128;   // partial-sum blocks of one call
constexpr int NOALLOC_MAX_STATES = HPSI_NOALLOC_MAX_STATES;
// partials [NOALLOC_BLOCKS][nst][4] followed by the result [nst][2]
constexpr size_t NOALLOC_DOUBLES =
    size_t(NOALLOC_BLOCKS) * NOALLOC_MAX_STATES * 4 + size_t(NOALLOC_MAX_STATES) * 2;

static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_DOUBLES];

constexpr int MAX_DEVICES = 64;
std::mutex g_mu;
double *g_scratch_addr[MAX_DEVICES] = {nullptr};

// Device address of the scratch array on the current device (set up once per
// device, with that device current).
hpsi_status scratch_address(double **out) {
  int dev = 0;
  HPSI_TRY_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= MAX_DEVICES) {
    set_error("hpsi_nrm2_noalloc: device ordinal out of range");
    return HPSI_ERR_UNSUPPORTED;
  }
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_addr[dev]) {
    void *ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess) {
      set_error(std::string("hpsi_nrm2_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      return HPSI_ERR_CUDA;
    }
    g_scratch_addr[dev] = static_cast<double *>(ptr);
  }
  *out = g_scratch_addr[dev];
  return HPSI_OK;
}

}  // namespace

}  // namespace hpsi

using namespace hpsi;

extern "C" hpsi_status hpsi_nrm2_noalloc(int32_t np, double vol_pp, const hpsi_batch *psi, double *out,
                                         void *stream) {
  if (!psi || !psi->ptr || !out || np < 1 || !(vol_pp > 0.0)) {
    set_error("hpsi_nrm2_noalloc: bad argument");
    return HPSI_ERR_ARG;
  }
  if (psi->dtype != HPSI_C128 && psi->dtype != HPSI_C64) {
    set_error("hpsi_nrm2_noalloc: unknown dtype");
    return HPSI_ERR_ARG;
  }
  if (psi->nst < 1 || psi->ld < psi->nst || psi->npts < np) {
    set_error("hpsi_nrm2_noalloc: need 1 <= nst <= ld and npts >= np");
    return HPSI_ERR_ARG;
  }
  if (psi->nst > NOALLOC_MAX_STATES) {
    set_error("hpsi_nrm2_noalloc: " + std::to_string(psi->nst) + " states exceed the maximum of " +
              std::to_string(NOALLOC_MAX_STATES));
    return HPSI_ERR_ARG;
  }
  if (!is_device_ptr(psi->ptr)) {
    set_error("hpsi_nrm2_noalloc: device batch expected");
    return HPSI_ERR_ARG;
  }
  double *scratch = nullptr;
  hpsi_status s = scratch_address(&scratch);
  if (s) return s;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int nst = psi->nst;
  double *partial = scratch;  // every entry is rewritten by the call: no clearing
  double *res = scratch + size_t(NOALLOC_BLOCKS) * nst * 4;
  if (psi->dtype == HPSI_C128)
    s = launch_state_sum<double>(0, static_cast<const double *>(psi->ptr), psi->ld, nullptr, 0, np, nst, partial,
                                 NOALLOC_BLOCKS, vol_pp, 1, res, st);
  else
    s = launch_state_sum<float>(0, static_cast<const float *>(psi->ptr), psi->ld, nullptr, 0, np, nst, partial,
                                NOALLOC_BLOCKS, vol_pp, 1, res, st);
  if (s) return s;
  // the result pairs (norm, 0) are strided by 2: copy the norms out
  HPSI_TRY_CUDA(cudaMemcpy2DAsync(out, sizeof(double), res, 2 * sizeof(double), sizeof(double), size_t(nst),
                                  cudaMemcpyDefault, st));
  if (!is_device_ptr(out)) HPSI_TRY_CUDA(cudaStreamSynchronize(st));
  return HPSI_OK;
}
