// Register-blocked real-lane stencil pass (see stencil_blk.cu).
#pragma once

#include "stencil.cuh"

namespace hpsi {

// Cell tile of one CTA: 16 x 8 (work items over 16 x 8 tiles).
constexpr int BLK_TILE_X = 16;
constexpr int BLK_TILE_Y = 8;

// Complex states per chunk of the blocked pass (FP64 8, FP32 16).
template <typename T>
int blk_chunk_states();

// The blocked pass serves a call when its chunk divides ld and the batches
// are 16-byte aligned.
template <typename T>
bool blk_pass_eligible(const PassArgs &a, long long ld);

// a.chunks = ld / blk_chunk_states<T>(); a.items over 16 x 8 tiles;
// observables, when requested, are written per item.  rx x ry: cells per
// thread; cplx: a thread owns a complex state (else one real lane); group:
// planes per unrolled group of the z march (1 or 3).
template <typename T>
hpsi_status launch_pass_blk(const PassArgs &a, int rx, int ry, int cplx, int group, cudaStream_t st);

// Grouped systems in one persistent launch (Horner passes): every system's
// arguments built with the blocked shape (items over 16 x 8 tiles).
template <typename T>
hpsi_status launch_pass_blk_group(const GroupArgs &g, int rx, int ry, int cplx, int group, int num_sms,
                                  cudaStream_t st);

}  // namespace hpsi
