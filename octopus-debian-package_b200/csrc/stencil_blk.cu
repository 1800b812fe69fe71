// Fused H.psi stencil pass with register-blocked real lanes (sm_100a).
//
// Same arithmetic and pass modes as the one-complex-per-thread pass in
// stencil.cu, with a division of work that cuts shared-memory reads per
// output: a CTA of 256 threads owns a 16 x 8 cell tile and one chunk of
// 128 bytes of every cell row (FP64 8 complex states, FP32 16); each thread
// owns one real lane (the re or im part of one state) of an RX x RY block of
// cells (FP64 2 x 4, FP32 4 x 4) and keeps nine running z sums per cell in
// registers.  Per output it reads 1 + 8/RX + 8/RY values from shared memory
// (7 FP64, 5 FP32) instead of 13 double2.  The Horner update takes the other
// part of h = (H u)(r) from the neighbouring lane by one shuffle.
//
// Halo planes (24 x 16 cells) are gathered through the load map into an
// NBUF-deep ring with 16-byte cp.async copies (eight threads per 128-byte cell
// chunk, so every warp copies four whole chunks); zero-boundary cells are
// stored as zeros and Bloch-phase images are multiplied on load.  The load
// map of each plane and the output rows four planes below travel in a side
// ring two stage rounds ahead of the data, so every gather knows its rows
// when it is issued.  One __syncthreads per plane (or, PassShape::mb, a full
// and an empty mbarrier per stage: a warp may run a plane ahead).
//
// A TMA tile::gather4 fill of the same 128-byte chunks (one producer warp,
// mbarrier hand-over) was measured 3x slower than this form on the same
// tiles: the bulk-copy engine does not keep enough 128-byte requests in
// flight per SM, while 256 threads issuing cp.async do.
//
// Reference semantics as in stencil.cu: X(nl_operator_operate_batch)
// (src/grid/nl_operator_inc.F90:21-130), the local potential
// (src/hamiltonian/hamiltonian_elec_base_inc.F90:233-242) and the Taylor
// axpys (src/electrons/exponential.F90:738-746).
#include <string>

#include "stencil_blk_impl.cuh"

namespace hpsi {

using namespace blk;

namespace blk {
// instantiated in stencil_blk_shapes.cu, one object per shape
extern template hpsi_status launch_blk_u<double, 9, 2, 2, false, 8, 128>(const PassArgs &, const CUtensorMap *, cudaStream_t);
extern template hpsi_status launch_blk_u<double, 3, 2, 2, false, 8, 128>(const PassArgs &, const CUtensorMap *, cudaStream_t);
extern template hpsi_status launch_blk_u<double, 9, 2, 2, true, 8, 128>(const PassArgs &, const CUtensorMap *, cudaStream_t);
extern template hpsi_status launch_blk_u<double, 9, 1, 4, false, 8, 64>(const PassArgs &, const CUtensorMap *, cudaStream_t);
extern template hpsi_status launch_blk_u<double, 9, 1, 4, false, 16, 64>(const PassArgs &, const CUtensorMap *, cudaStream_t);
extern template hpsi_status launch_blk_u<float, 9, 2, 2, true, 8, 128>(const PassArgs &, const CUtensorMap *, cudaStream_t);
extern template hpsi_status launch_blk_u<float, 3, 2, 2, true, 8, 128>(const PassArgs &, const CUtensorMap *, cudaStream_t);
extern template hpsi_status launch_blk_u<float, 1, 2, 4, false, 8, 128>(const PassArgs &, const CUtensorMap *, cudaStream_t);
extern template hpsi_status launch_blk_u<float, 9, 1, 4, true, 8, 64>(const PassArgs &, const CUtensorMap *, cudaStream_t);
extern template hpsi_status launch_blk_u<float, 9, 1, 4, true, 16, 64>(const PassArgs &, const CUtensorMap *, cudaStream_t);
extern template hpsi_status launch_blk_u<double, 9, 2, 2, false, 8, 128, true>(const PassArgs &, const CUtensorMap *,
                                                                               cudaStream_t);
extern template hpsi_status launch_blk_u<float, 9, 2, 2, true, 8, 128, true>(const PassArgs &, const CUtensorMap *,
                                                                             cudaStream_t);
extern template hpsi_status launch_blk_u<double, 9, 2, 2, false, 8, 128, false, true>(const PassArgs &,
                                                                                      const CUtensorMap *,
                                                                                      cudaStream_t);
extern template hpsi_status launch_blk_u<float, 9, 2, 2, true, 8, 128, false, true>(const PassArgs &,
                                                                                    const CUtensorMap *,
                                                                                    cudaStream_t);
}  // namespace blk


template <typename T>
hpsi_status launch_pass_blk_group(const GroupArgs &g, const PassShape &s, int num_sms, cudaStream_t st) {
  if (g.nunits == 0) return HPSI_OK;
  const int grid = std::min(g.nunits, num_sms);
  const int cb = shape_cb<T>(s);
  if constexpr (sizeof(T) == 8) {
    if (!s.cplx && s.rx == 2 && s.ry == 2 && s.unroll == 9 && s.ty == 8 && cb == 128)
      return launch_blk_group_v<T, 9, 2, 2, false, 8, 128>(g, grid, st);
  } else {
    if (s.cplx && s.rx == 2 && s.ry == 2 && s.unroll == 9 && s.ty == 8 && cb == 128)
      return launch_blk_group_v<T, 9, 2, 2, true, 8, 128>(g, grid, st);
  }
  set_error("launch_pass_blk_group: no kernel for this cell block");
  return HPSI_ERR_UNSUPPORTED;
}
template hpsi_status launch_pass_blk_group<double>(const GroupArgs &, const PassShape &, int, cudaStream_t);
template hpsi_status launch_pass_blk_group<float>(const GroupArgs &, const PassShape &, int, cudaStream_t);

template <typename T>
int blk_chunk_states() {
  return 128 / int(sizeof(T)) / 2;
}

template <typename T>
bool blk_pass_eligible(const PassArgs &a, long long ld, int sc) {
  if (ld % sc != 0) return false;
  if (reinterpret_cast<uintptr_t>(a.in) % 16 != 0 || reinterpret_cast<uintptr_t>(a.out) % 16 != 0) return false;
  if ((a.mode == PASS_HORNER || a.obs) && reinterpret_cast<uintptr_t>(a.psi0) % 16 != 0) return false;
  if ((2 * a.in_ld * sizeof(T)) % 16 != 0 || (2 * a.psi0_ld * sizeof(T)) % 16 != 0) return false;
  return true;
}

// Instantiated blocks (512 threads each):
//   128-byte chunks, 16 x 8 tiles: FP64 2 x 2 real lanes (groups of 9 or 3)
//     or complex states (9); FP32 2 x 2 complex states with packed
//     multiply-adds (9 or 3) or 2 x 4 real lanes (1);
//   64-byte chunks, 16 x 16 tiles (halo 2.25x instead of 3x): 1 x 4 cells,
//     FP64 real lanes, FP32 complex states (groups of 9);
//   64-byte chunks, 16 x 8 tiles, 1 x 4 cells, 256 threads and two CTAs per
//     SM (faster on small meshes: twice the CTAs per state chunk).
// Tensor map of a pass input for the TMA fill: [in_rows][2 in_ld] elements of
// the storage type, box 8 rows x one 128-byte chunk, no swizzle, zero fill
// outside (never reached: only runs of eight existing rows are copied).
// cuTensorMapEncodeTiled comes through the runtime's driver entry point.
template <typename T>
static hpsi_status encode_input_map(const PassArgs &a, CUtensorMap *tm) {
  using enc_fn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                              const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                              CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
  static enc_fn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<enc_fn>(p);
  });
  if (!fn) {
    set_error("launch_pass_blk: cuTensorMapEncodeTiled unavailable");
    return HPSI_ERR_UNSUPPORTED;
  }
  const cuuint64_t dims[2] = {cuuint64_t(2 * a.in_ld), cuuint64_t(a.in_rows)};
  const cuuint64_t strides[1] = {cuuint64_t(2 * a.in_ld) * sizeof(T)};
  const cuuint32_t box[2] = {cuuint32_t(128 / sizeof(T)), 8};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = fn(tm, sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
                        const_cast<void *>(a.in), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("launch_pass_blk: cuTensorMapEncodeTiled failed (" + std::to_string(int(r)) + ")");
    return HPSI_ERR_CUDA;
  }
  return HPSI_OK;
}

template <typename T>
hpsi_status launch_pass_blk(const PassArgs &a, const PassShape &s, cudaStream_t st) {
  if (a.nitems == 0) return HPSI_OK;
  const int cb = shape_cb<T>(s), g = s.unroll;
  if (s.tma) {
    // TMA fill: the default cell blocks (FP64 2 x 2 real lanes, FP32 2 x 2
    // complex states), 16 x 8 tiles, 128-byte chunks, no Bloch phase
    if (s.ty != 8 || cb != 128 || s.rx != 2 || s.ry != 2 || g != 9 || a.phase_corr || !a.seg_mask ||
        s.cplx != (sizeof(T) == 8 ? 0 : 1) || a.in_rows <= 0) {
      set_error("launch_pass_blk: no TMA-fill kernel for this pass");
      return HPSI_ERR_UNSUPPORTED;
    }
    alignas(64) CUtensorMap tm;
    hpsi_status r = encode_input_map<T>(a, &tm);
    if (r) return r;
    if constexpr (sizeof(T) == 8)
      return launch_blk_u<T, 9, 2, 2, false, 8, 128, true>(a, &tm, st);
    else
      return launch_blk_u<T, 9, 2, 2, true, 8, 128, true>(a, &tm, st);
  }
  if (s.mma) {
    // FP64 only: in-plane arms as DMMA banded products, 8-state chunks
    if (sizeof(T) != 8 || cb != 128 || s.ty != 8) {
      set_error("launch_pass_blk: the tensor-core pass is FP64 with 8-state chunks");
      return HPSI_ERR_UNSUPPORTED;
    }
    return launch_pass_mma(a, st);
  }
  if (s.mb) {
    // mbarrier hand-over of the stages: the default cell blocks
    if (s.ty != 8 || cb != 128 || s.rx != 2 || s.ry != 2 || g != 9 || s.cplx != (sizeof(T) == 8 ? 0 : 1)) {
      set_error("launch_pass_blk: no mbarrier-pipelined kernel for this cell block");
      return HPSI_ERR_UNSUPPORTED;
    }
    if constexpr (sizeof(T) == 8)
      return launch_blk_u<T, 9, 2, 2, false, 8, 128, false, true>(a, nullptr, st);
    else
      return launch_blk_u<T, 9, 2, 2, true, 8, 128, false, true>(a, nullptr, st);
  }
  if (s.ty == 8 && cb == 128) {
    if constexpr (sizeof(T) == 8) {
      if (!s.cplx && s.rx == 2 && s.ry == 2 && g == 9) return launch_blk_u<T, 9, 2, 2, false, 8, 128>(a, nullptr, st);
      if (!s.cplx && s.rx == 2 && s.ry == 2 && g == 3) return launch_blk_u<T, 3, 2, 2, false, 8, 128>(a, nullptr, st);
      if (s.cplx && s.rx == 2 && s.ry == 2 && g == 9) return launch_blk_u<T, 9, 2, 2, true, 8, 128>(a, nullptr, st);
    } else {
      if (s.cplx && s.rx == 2 && s.ry == 2 && g == 9) return launch_blk_u<T, 9, 2, 2, true, 8, 128>(a, nullptr, st);
      if (s.cplx && s.rx == 2 && s.ry == 2 && g == 3) return launch_blk_u<T, 3, 2, 2, true, 8, 128>(a, nullptr, st);
      if (!s.cplx && s.rx == 2 && s.ry == 4 && g == 1) return launch_blk_u<T, 1, 2, 4, false, 8, 128>(a, nullptr, st);
    }
  } else if (s.ty == 8 && cb == 64 && s.rx == 1 && s.ry == 4 && g == 9) {
    // 256-thread blocks, two CTAs per SM
    if constexpr (sizeof(T) == 8) {
      if (!s.cplx) return launch_blk_u<T, 9, 1, 4, false, 8, 64>(a, nullptr, st);
    } else {
      if (s.cplx) return launch_blk_u<T, 9, 1, 4, true, 8, 64>(a, nullptr, st);
    }
  } else if (s.ty == 16 && cb == 64 && s.rx == 1 && s.ry == 4 && g == 9) {
    if constexpr (sizeof(T) == 8) {
      if (!s.cplx) return launch_blk_u<T, 9, 1, 4, false, 16, 64>(a, nullptr, st);
    } else {
      if (s.cplx) return launch_blk_u<T, 9, 1, 4, true, 16, 64>(a, nullptr, st);
    }
  }
  set_error("launch_pass_blk: no kernel for this cell block");
  return HPSI_ERR_UNSUPPORTED;
}

template int blk_chunk_states<double>();
template int blk_chunk_states<float>();
template bool blk_pass_eligible<double>(const PassArgs &, long long, int);
template bool blk_pass_eligible<float>(const PassArgs &, long long, int);
template hpsi_status launch_pass_blk<double>(const PassArgs &, const PassShape &, cudaStream_t);
template hpsi_status launch_pass_blk<float>(const PassArgs &, const PassShape &, cudaStream_t);

}  // namespace hpsi
