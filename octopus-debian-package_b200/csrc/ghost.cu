// Ghost-row exchange of a domain-parallel mesh: the device side of
// X(ghost_update_batch_start) / X(ghost_update_batch_finish)
// (src/grid/boundaries_inc.F90:57-231).  A partition's rows are its local
// points, then its ghost rows grouped by source partition (ghost_rdispls /
// ghost_rcounts), then its boundary points, as in par_vec_t.  The sender packs
// the rows that its neighbours hold as ghosts into one contiguous buffer
// through the send map (the reference's ghost_reorder kernel); the receiver
// takes each message straight into its ghost rows when the batch rows are
// contiguous (ld == nst), or through hpsi_ghost_unpack otherwise.  The
// transport between the two (NCCL send/recv over NVLink) is the caller's.
//
// One warp per row; lanes copy 16-byte (complex128) or 8-byte (complex64)
// elements, so a row of nst states moves in ceil(nst / 32) coalesced rounds.
// Entries of the maps outside [0, npts) are skipped (the maps come from the
// partitioner, which checks them on the host).
#include "api_internal.cuh"

namespace hpsi {
namespace {

template <typename V>
__global__ void __launch_bounds__(256) ghost_pack_kernel(const V *__restrict__ psi, long long ld, int npts, int nst,
                                                        const int *__restrict__ map, int count,
                                                        V *__restrict__ out) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= count) return;
  const int row = map[w];
  if (row < 0 || row >= npts) return;
  const V *src = psi + (long long)row * ld;
  V *dst = out + (long long)w * nst;
  for (int s = lane; s < nst; s += 32) dst[s] = src[s];
}

template <typename V>
__global__ void __launch_bounds__(256) ghost_unpack_kernel(const V *__restrict__ in, const int *__restrict__ pos,
                                                          int count, V *__restrict__ psi, long long ld, int npts,
                                                          int nst) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= count) return;
  const int row = pos[w];
  if (row < 0 || row >= npts) return;
  const V *src = in + (long long)w * nst;
  V *dst = psi + (long long)row * ld;
  for (int s = lane; s < nst; s += 32) dst[s] = src[s];
}

hpsi_status check_ghost_args(const char *fn, const hpsi_batch *b, const int32_t *map, int32_t count,
                             const void *buf) {
  if (!b || count < 0 || (count > 0 && (!map || !buf || !b->ptr)) || b->nst < 1 || b->ld < b->nst ||
      b->npts < 0 || (b->dtype != HPSI_C128 && b->dtype != HPSI_C64)) {
    set_error(std::string(fn) + ": bad argument");
    return HPSI_ERR_ARG;
  }
  if (count > 0 && (!is_device_ptr(b->ptr) || !is_device_ptr(map) || !is_device_ptr(buf))) {
    set_error(std::string(fn) + ": batch, map and buffer must be device memory");
    return HPSI_ERR_ARG;
  }
  return HPSI_OK;
}

}  // namespace
}  // namespace hpsi

using namespace hpsi;

extern "C" hpsi_status hpsi_ghost_pack(const hpsi_batch *psi, const int32_t *sendmap, int32_t count, void *sendbuf,
                                       void *stream) {
  hpsi_status s = check_ghost_args("hpsi_ghost_pack", psi, sendmap, count, sendbuf);
  if (s || count == 0) return s;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const unsigned grid = unsigned((count + 7) / 8);
  if (psi->dtype == HPSI_C128)
    ghost_pack_kernel<double2><<<grid, 256, 0, st>>>(static_cast<const double2 *>(psi->ptr), psi->ld, psi->npts,
                                                     psi->nst, sendmap, count, static_cast<double2 *>(sendbuf));
  else
    ghost_pack_kernel<float2><<<grid, 256, 0, st>>>(static_cast<const float2 *>(psi->ptr), psi->ld, psi->npts,
                                                    psi->nst, sendmap, count, static_cast<float2 *>(sendbuf));
  HPSI_CHECK_LAUNCH();
  return HPSI_OK;
}

extern "C" hpsi_status hpsi_ghost_unpack(const void *recvbuf, const int32_t *pos, int32_t count, hpsi_batch *psi,
                                         void *stream) {
  hpsi_status s = check_ghost_args("hpsi_ghost_unpack", psi, pos, count, recvbuf);
  if (s || count == 0) return s;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const unsigned grid = unsigned((count + 7) / 8);
  if (psi->dtype == HPSI_C128)
    ghost_unpack_kernel<double2><<<grid, 256, 0, st>>>(static_cast<const double2 *>(recvbuf), pos, count,
                                                       static_cast<double2 *>(psi->ptr), psi->ld, psi->npts,
                                                       psi->nst);
  else
    ghost_unpack_kernel<float2><<<grid, 256, 0, st>>>(static_cast<const float2 *>(recvbuf), pos, count,
                                                      static_cast<float2 *>(psi->ptr), psi->ld, psi->npts, psi->nst);
  HPSI_CHECK_LAUNCH();
  return HPSI_OK;
}
