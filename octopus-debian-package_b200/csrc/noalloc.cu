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
// the symbol itself: its device address is looked up with
// cudaGetSymbolAddress once per CUDA context (the module, and with it the
// array, is loaded separately into every context, so a device ordinal is not
// enough to name it when a host application creates its own contexts) and
// that address is handed to the kernels.
#include <mutex>
#include <string>
#include <utility>
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

std::mutex g_mu;
// (context, device address of the array in it); a handful of entries at most
std::vector<std::pair<void *, double *>> g_scratch_addr;

// The current driver context, through the runtime's driver entry point (the
// library does not link the driver library itself).  nullptr when no context
// is current yet.
hpsi_status current_context(void **ctx) {
  using get_fn = int (*)(void **);
  static get_fn fn = nullptr;
  static std::once_flag once;
  static cudaError_t lookup = cudaSuccess;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    lookup = cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q);
    if (lookup == cudaSuccess && q == cudaDriverEntryPointSuccess) fn = reinterpret_cast<get_fn>(p);
  });
  if (!fn) {
    set_error("hpsi_nrm2_noalloc: cuCtxGetCurrent is not available from the driver");
    return HPSI_ERR_CUDA;
  }
  *ctx = nullptr;
  if (fn(ctx) != 0) {
    set_error("hpsi_nrm2_noalloc: cuCtxGetCurrent failed");
    return HPSI_ERR_CUDA;
  }
  return HPSI_OK;
}

// Device address of the scratch array in the current context (looked up once
// per context, with that context current).
hpsi_status scratch_address(double **out) {
  void *ctx = nullptr;
  hpsi_status s = current_context(&ctx);
  if (s) return s;
  std::lock_guard<std::mutex> lk(g_mu);
  if (ctx)
    for (auto &e : g_scratch_addr)
      if (e.first == ctx) {
        *out = e.second;
        return HPSI_OK;
      }
  void *ptr = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
  if (e != cudaSuccess) {
    set_error(std::string("hpsi_nrm2_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    return HPSI_ERR_CUDA;
  }
  // with no context current before, the runtime has just made the device's
  // primary context current: key the entry on it
  if (!ctx) {
    s = current_context(&ctx);
    if (s) return s;
  }
  if (ctx) g_scratch_addr.emplace_back(ctx, static_cast<double *>(ptr));
  *out = static_cast<double *>(ptr);
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
