// Explicit instantiations of the register-blocked pass, one cell-block shape
// per object: the Makefile compiles this file once per HPSI_BLK_SHAPE
// (0..13), so that the shapes, each a 9-plane unrolled kernel in five modes,
// compile in parallel.  The list matches the extern declarations in
// stencil_blk.cu.
#include "stencil_blk_impl.cuh"

#ifndef HPSI_BLK_SHAPE
#error "HPSI_BLK_SHAPE must be defined"
#endif

namespace hpsi {
namespace blk {

#if HPSI_BLK_SHAPE == 0
template hpsi_status launch_blk_u<double, 9, 2, 2, false, 8, 128>(const PassArgs &, const CUtensorMap *, cudaStream_t);
#elif HPSI_BLK_SHAPE == 1
template hpsi_status launch_blk_u<double, 3, 2, 2, false, 8, 128>(const PassArgs &, const CUtensorMap *, cudaStream_t);
#elif HPSI_BLK_SHAPE == 2
template hpsi_status launch_blk_u<double, 9, 2, 2, true, 8, 128>(const PassArgs &, const CUtensorMap *, cudaStream_t);
#elif HPSI_BLK_SHAPE == 3
template hpsi_status launch_blk_u<double, 9, 1, 4, false, 8, 64>(const PassArgs &, const CUtensorMap *, cudaStream_t);
#elif HPSI_BLK_SHAPE == 4
template hpsi_status launch_blk_u<double, 9, 1, 4, false, 16, 64>(const PassArgs &, const CUtensorMap *, cudaStream_t);
#elif HPSI_BLK_SHAPE == 5
template hpsi_status launch_blk_u<float, 9, 2, 2, true, 8, 128>(const PassArgs &, const CUtensorMap *, cudaStream_t);
#elif HPSI_BLK_SHAPE == 6
template hpsi_status launch_blk_u<float, 3, 2, 2, true, 8, 128>(const PassArgs &, const CUtensorMap *, cudaStream_t);
#elif HPSI_BLK_SHAPE == 7
template hpsi_status launch_blk_u<float, 1, 2, 4, false, 8, 128>(const PassArgs &, const CUtensorMap *, cudaStream_t);
#elif HPSI_BLK_SHAPE == 8
template hpsi_status launch_blk_u<float, 9, 1, 4, true, 8, 64>(const PassArgs &, const CUtensorMap *, cudaStream_t);
#elif HPSI_BLK_SHAPE == 9
template hpsi_status launch_blk_u<float, 9, 1, 4, true, 16, 64>(const PassArgs &, const CUtensorMap *, cudaStream_t);
#elif HPSI_BLK_SHAPE == 10
template hpsi_status launch_blk_u<double, 9, 2, 2, false, 8, 128, true>(const PassArgs &, const CUtensorMap *, cudaStream_t);
#elif HPSI_BLK_SHAPE == 11
template hpsi_status launch_blk_u<float, 9, 2, 2, true, 8, 128, true>(const PassArgs &, const CUtensorMap *, cudaStream_t);
#elif HPSI_BLK_SHAPE == 12
template hpsi_status launch_blk_u<double, 9, 2, 2, false, 8, 128, false, true>(const PassArgs &, const CUtensorMap *,
                                                                               cudaStream_t);
#elif HPSI_BLK_SHAPE == 13
template hpsi_status launch_blk_u<float, 9, 2, 2, true, 8, 128, false, true>(const PassArgs &, const CUtensorMap *,
                                                                             cudaStream_t);
#else
#error "unknown HPSI_BLK_SHAPE"
#endif

}  // namespace blk
}  // namespace hpsi
