// Batched swept phases: many independent instances (uneven grid sizes) advance
// together, one launch per phase for all of them.
//
// Every instance has two descriptors (SweptArgs for even and odd
// half-cycles: base buffers swapped, prism bands offset by 0 or bs/2) and
// contributes its (band, segment) units to one flat unit table of
// (instance, unit) pairs.  A batched launch maps warp / CTA g to table entry g
// and runs the same body as the single-instance kernel.  All instances share
// the blocksize, so they share the levels per half-cycle and the shared-memory
// layout.  The launches of a whole run are captured into one CUDA graph.
#pragma once
#include "heat_fast.cuh"
#include "seam_fast.cuh"
#include "swept.cuh"

namespace psb {

// Descriptors [instance][role][parity]: role 0 for the prism stream and the
// y-bridge, role 1 for the gap stream and the octahedron (their y-faces live in
// a second buffer, because the gap runs beside the y-bridge).
//
// The register heat kernels (one warp per table entry) copy their entry's
// descriptor into shared memory, kDescBytes per warp at the start of the
// dynamic shared memory, and the bodies read the fields from there as the
// single-instance kernels read their parameter-bank copy: a copy in
// registers spilled 84-200 bytes per thread in the bs-32 streams (256 heat
// instances of 128-2048², 1000 steps: 0.703 -> 0.615 s).  The generic
// kernels keep a copy in registers (batch_args): for Euler the shared copy
// measured no better.
constexpr int kDescBytes = (int)((sizeof(SweptArgs) + 15) / 16 * 16);
static_assert(sizeof(SweptArgs) % 8 == 0, "the descriptor copies in 8-byte words");

// The generic kernels' register copy, with this launch's levels and first
// level.
template <bool GAP>
__device__ __forceinline__ void batch_args(const SweptArgs* __restrict__ desc, int inst,
                                           int parity, int H, long long L0, SweptArgs& a)
{
    a = desc[4 * inst + 2 * (GAP ? 1 : 0) + parity];
    a.H = H;
    a.L0 = L0;
}

// Threads t of [0, nt) copy descriptor `inst` into `slot`; after the callers'
// barrier, one of them (t == 0) sets this launch's levels and first level,
// and a second barrier publishes the copy.
template <bool GAP>
__device__ __forceinline__ void batch_desc_copy(const SweptArgs* __restrict__ desc, int inst,
                                                int parity, SweptArgs* slot, int t, int nt)
{
    const unsigned long long* src = reinterpret_cast<const unsigned long long*>(
        desc + 4 * inst + 2 * (GAP ? 1 : 0) + parity);
    unsigned long long* dst = reinterpret_cast<unsigned long long*>(slot);
    for (int w = t; w < (int)(sizeof(SweptArgs) / 8); w += nt) dst[w] = src[w];
}

template <int BX, bool GAP>
__global__ void __launch_bounds__(32 * kFastWarps, 3)
    heat_stream_fast_batch(const SweptArgs* __restrict__ desc, const int2* __restrict__ units,
                           int nunits, int parity, int H, long long L0)
{
    extern __shared__ double sm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = blockIdx.x * kFastWarps + warp;
    if (g >= nunits) return;  // whole warp
    const int2 u = units[g];
    SweptArgs* slot = reinterpret_cast<SweptArgs*>(reinterpret_cast<char*>(sm) + warp * kDescBytes);
    batch_desc_copy<GAP>(desc, u.x, parity, slot, lane, 32);
    __syncwarp();
    if (lane == 0) {
        slot->H = H;
        slot->L0 = L0;
    }
    __syncwarp();
    const SweptArgs& a = *slot;
    double* base = sm + kFastWarps * kDescBytes / 8;
    heat_fast_body<BX, GAP>(a, seg_geom(a, u.y), u.y,
                            base + (size_t)warp * heat_fast_warp_doubles<BX>(a.Hmax));
}

// The register-resident heat seams (seam_fast.cuh) over the unit table: one
// warp per (instance, unit).  GAP selects the octahedron (role-1 descriptors).
template <int BX, bool GAP>
__global__ void __launch_bounds__(32 * kSeamWarps)
    heat_seam_fast_batch(const SweptArgs* __restrict__ desc, const int2* __restrict__ units,
                         int nunits, int parity, int H, long long L0)
{
    extern __shared__ double sm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = blockIdx.x * kSeamWarps + warp;
    if (g >= nunits) return;  // whole warp
    const int2 u = units[g];
    SweptArgs* slot = reinterpret_cast<SweptArgs*>(reinterpret_cast<char*>(sm) + warp * kDescBytes);
    batch_desc_copy<GAP>(desc, u.x, parity, slot, lane, 32);
    __syncwarp();
    if (lane == 0) {
        slot->H = H;
        slot->L0 = L0;
    }
    __syncwarp();
    const SweptArgs& a = *slot;
    double* ys = sm + kSeamWarps * kDescBytes / 8 + (size_t)warp * yseam_warp_doubles<BX>(a.Hmax);
    if constexpr (GAP)
        heat_oseam_body<BX>(a, u.y, ys);
    else
        heat_yseam_body<BX>(a, u.y, ys);
}

// The generic batched kernels hold the descriptor fields in registers (the
// single-instance kernels read them from the parameter bank), so they are
// capped at the single-instance register budget to keep two stream CTAs (four
// seam CTAs) per SM.
template <class Eq, int ITS, int W, bool GAP, int NT>
__global__ void __launch_bounds__(NT, 2)
    stream_batch(const SweptArgs* __restrict__ desc, const int2* __restrict__ units, int parity,
                 int H, long long L0)
{
    extern __shared__ double sm[];
    const int2 u = units[blockIdx.x];
    SweptArgs a;
    batch_args<GAP>(desc, u.x, parity, H, L0, a);
    stream_body<Eq, ITS, W, GAP, NT>(a, u.y, sm);
}

template <class Eq, int ITS, bool GAP, int NT>
__global__ void __launch_bounds__(NT, 4)
    seam_batch(const SweptArgs* __restrict__ desc, const int2* __restrict__ units, int parity,
               int H, long long L0)
{
    extern __shared__ double sm[];
    const int2 u = units[blockIdx.x];
    SweptArgs a;
    batch_args<GAP>(desc, u.x, parity, H, L0, a);
    seam_body<Eq, ITS, GAP, NT>(a, u.y, sm);
}

}  // namespace psb
