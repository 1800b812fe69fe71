// Register-blocked real-lane stencil pass (see stencil_blk.cu).
#pragma once

#include "stencil.cuh"

namespace hpsi {

// Cell tiles of one CTA: 16 x 8 (128-byte chunks) or 16 x 16 (64-byte chunks).
constexpr int BLK_TILE_X = 16;

// Complex states per 128-byte chunk of the blocked pass (FP64 8, FP32 16).
template <typename T>
int blk_chunk_states();

// The blocked pass serves a call when its chunk (sc complex states) divides
// ld and the batches are 16-byte aligned.
template <typename T>
bool blk_pass_eligible(const PassArgs &a, long long ld, int sc);

// a.chunks = ld / shape.sc; a.items over 16 x shape.ty tiles; observables,
// when requested, are written per item.  The shape names the cell block
// (rx x ry), the element (cplx: a complex state per thread, else one real
// lane) and the planes per unrolled group (unroll).
template <typename T>
hpsi_status launch_pass_blk(const PassArgs &a, const PassShape &shape, cudaStream_t st);

// FP64 pass with the in-plane arms on the FP64 tensor cores (stencil_mma.cu):
// 16 x 8 tiles, chunks of 8 complex states, no fused density.
hpsi_status launch_pass_mma(const PassArgs &a, cudaStream_t st);

// Grouped systems in one persistent launch (Horner passes): every system's
// arguments built with the blocked shape (items over 16 x 8 tiles).
template <typename T>
hpsi_status launch_pass_blk_group(const GroupArgs &g, const PassShape &shape, int num_sms, cudaStream_t st);

}  // namespace hpsi
