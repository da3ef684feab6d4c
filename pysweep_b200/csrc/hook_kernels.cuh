// Kernels around a user step hook, compiled at run time (NVRTC, sm_100a) with
// the hook's source.  Host side: hook.cuh.
//
// The reference includes the plugin's
//     __device__ void step(double* shared_state, int idx, int globalTimeStep)
// textually into its phase kernels (pysweep/core/pysweep.cu:25,
// pysweep/core/io.py:146-155) and gives it the framework constants VARS,
// TIMES, MPSS, MOSS, NV, OPS, ITS, SX, SY as __constant__ ints
// (pysweep/core/pysweep.cu:12-20): the hook reads variable v of the cell at
// idx + v*VARS, its neighbours at idx +- SY (rows) and idx +- 1 (columns),
// the previous level at idx - TIMES and writes the next one at idx + TIMES.
//
// Here the hook runs inside the same swept phases as the built-in equations
// (stream_body and seam_body of swept.cuh, with the LINEAR slot layout that
// keeps the previous, current and next level at one stride) and inside a
// tiled standard step.  Each kernel kind has its own tile geometry, so the
// generated source includes the hook once per kind, in the namespaces
// psh_stream, psh_seam and psh_std, each with its own framework constants
// (set by the host before every run) and its own copy of the hook's
// __constant__ globals (set together by name).  The prelude defines
// PSH_OPS, PSH_ITS, PSH_NV and the standard tile (PSH_STD_TR x PSH_STD_TC
// cells, PSH_STD_NT threads) before including this file.
#pragma once
#include "swept.cuh"

namespace psb {

// The hook as a built-in equation functor: u points at the cell of the
// current level; the next and previous levels sit TIMES elements after and
// before it in the tile (the namespace's layout guarantees this), so u is
// passed as the shared array with idx = 0.
struct HookStream {
    static constexpr int OPS = PSH_OPS;
    __device__ static __forceinline__ void step(const double* u, const double*, double*, const Nbr&,
                                                int gts, int, const EqParams&)
    {
        psh_stream::step(const_cast<double*>(u), 0, gts);
    }
};

struct HookSeam {
    static constexpr int OPS = PSH_OPS;
    __device__ static __forceinline__ void step(const double* u, const double*, double*, const Nbr&,
                                                int gts, int, const EqParams&)
    {
        psh_seam::step(const_cast<double*>(u), 0, gts);
    }
};

// Standard step tiles: kStdTR x kStdTC cells per CTA, with an OPS-cell
// periodic halo on every side, three slots (previous, current, next level) of
// [NV][kStdTR + 2 OPS][kStdTC + 2 OPS] doubles: TIMES = one slot,
// VARS = one variable plane, SY = one tile row.
constexpr int kStdTR = PSH_STD_TR, kStdTC = PSH_STD_TC, kStdNT = PSH_STD_NT;
constexpr int kStdR = kStdTR + 2 * PSH_OPS, kStdC = kStdTC + 2 * PSH_OPS;
constexpr int kStdSlot = PSH_NV * kStdR * kStdC;

}  // namespace psb

using psb::SweptArgs;

// The streams (UpPyramid / XBridge), TIMES = slot + OPS: level m's column k
// sits OPS columns right of level m-1's (the chunk's parallelogram).
#define PSH_STREAM(NAME, W, GAP)                                                                  \
    extern "C" __global__ void __launch_bounds__(256) NAME(SweptArgs a)                         \
    {                                                                                             \
        extern __shared__ double psh_sm[];                                                        \
        psb::stream_body<psb::HookStream, PSH_ITS, W, GAP, 256, true>(a, blockIdx.x, psh_sm);    \
    }
PSH_STREAM(psh_prism32, 32, false)
PSH_STREAM(psh_gap32, 32, true)
PSH_STREAM(psh_prism64, 64, false)
PSH_STREAM(psh_gap64, 64, true)
#undef PSH_STREAM

// The seams (YBridge / Octahedron), TIMES = one slot.
extern "C" __global__ void __launch_bounds__(128) psh_ybridge(SweptArgs a)
{
    extern __shared__ double psh_sm[];
    psb::seam_body<psb::HookSeam, PSH_ITS, false, 128, double, true>(a, blockIdx.x, psh_sm);
}

extern "C" __global__ void __launch_bounds__(128) psh_octahedron(SweptArgs a)
{
    extern __shared__ double psh_sm[];
    psb::seam_body<psb::HookSeam, PSH_ITS, true, 128, double, true>(a, blockIdx.x, psh_sm);
}

// One level of the standard decomposition (pysweep/core/pysweep.cu:259-275):
// the tile of the current and previous level with its periodic halo into
// shared memory, the hook on every cell, the next level back to the ring
// (and to a frame when one is due).
extern "C" __global__ void __launch_bounds__(psb::kStdNT)
    psh_standard(const double* __restrict__ cur, const double* __restrict__ prev,
                 double* __restrict__ out, double* __restrict__ frame, int nx, int ny, int gts)
{
    using namespace psb;
    constexpr int OPS = PSH_OPS, NV = PSH_NV;
    extern __shared__ double t[];  // previous, current, next: 3 * kStdSlot
    const int x0 = blockIdx.y * kStdTR, y0 = blockIdx.x * kStdTC;
    const size_t vs = (size_t)nx * ny;
    for (int e = threadIdx.x; e < 2 * kStdSlot; e += kStdNT) {
        const int s = e / kStdSlot, r = e % kStdSlot;
        const int v = r / (kStdR * kStdC), i = (r / kStdC) % kStdR, k = r % kStdC;
        const int x = wrap(x0 + i - OPS, nx), y = wrap(y0 + k - OPS, ny);
        const double* src = s == 0 ? prev : cur;
        cp_async8(t + e, src + v * vs + (size_t)x * ny + y);
    }
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
    for (int c = threadIdx.x; c < kStdTR * kStdTC; c += kStdNT) {
        const int i = c / kStdTC, k = c % kStdTC;
        if (x0 + i < nx && y0 + k < ny)
            psh_std::step(t, kStdSlot + (i + OPS) * kStdC + k + OPS, gts);
    }
    __syncthreads();
    for (int c = threadIdx.x; c < NV * kStdTR * kStdTC; c += kStdNT) {
        const int v = c / (kStdTR * kStdTC), i = (c / kStdTC) % kStdTR, k = c % kStdTC;
        if (x0 + i >= nx || y0 + k >= ny) continue;
        const double val = t[2 * kStdSlot + (v * kStdR + i + OPS) * kStdC + k + OPS];
        const size_t go = v * vs + (size_t)(x0 + i) * ny + y0 + k;
        out[go] = val;
        if (frame) frame[go] = val;
    }
}
