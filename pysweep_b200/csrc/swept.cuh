// Swept space-time engine.
//
// The reference decomposes the periodic domain into bs x bs blocks and runs,
// per half-cycle of MPSS levels, the phases UpPyramid -> YBridge -> (shift by
// bs/2 rows) -> XBridge -> Octahedron -> YBridge -> ... -> DownPyramid
// (pysweep/core/pysweep.cu:64-249, pysweep/core/functions.py:12-123).  After
// UpPyramid + YBridge every row band of height bs holds a "prism": level m is
// complete on rows [OPS*m, bs-OPS*m) of the band, for every column.  After
// XBridge + the Octahedron's down half the gap between two prisms is filled
// and levels 1..MPSS are complete everywhere; the Octahedron's up half starts
// the next prisms on bands shifted by bs/2.
//
// This engine keeps that structure with blocks of Bx rows x Wy columns
// (Bx = bs sets MPSS = Bx/(2*OPS)-1; Wy is a multiple of the chunk width W):
//
//  P  (prism)   UpPyramid of one block.  The block is streamed through shared
//               memory in W-column chunks; chunk c computes, at level m, the
//               parallelogram of columns [c*W-OPS*m, (c+1)*W-OPS*m), so only the
//               last 2*OPS columns of every level ("carry") pass from one chunk
//               to the next.  At the block's left/right column edges the level
//               shrinks by OPS per level, exactly as an up pyramid does.
//  Y  (seam)    YBridge centred on each block column edge: grows in y, shrinks
//               in x, fed by the two neighbours' edge columns (y-faces).
//  G  (gap)     XBridge of the band boundary: rows [hx-OPS*m, hx+OPS*m) around
//               the boundary (hx = Bx/2), streamed like P; the rows it reads
//               from the two prisms (x-faces) come from global memory.
//  O  (seam)    The Octahedron's down half at each gap/column-edge corner:
//               grows in both x and y.
//  The next half-cycle's P phase on bands shifted by hx is the Octahedron's up
//  half (and, in the last half-cycle, G + O form the DownPyramid).
//
// Between phases only these pass through global memory:
//   * the base levels (the last ITS complete levels; ping-pong bin/bout),
//   * x-faces: 2*OPS rows at the top and bottom of every prism level,
//   * y-faces: 2*OPS columns at the left/right edge of every stream level.
// Every cell of every level is computed exactly once, by exactly the same
// per-cell function as the standard decomposition, so swept and standard
// results are bit-identical.
#pragma once
#ifndef __CUDACC_RTC__  // run-time compilation (user step hooks) has no host headers
#include <cuda_runtime.h>
#include <stdint.h>
#endif

#include "equations.cuh"

namespace psb {

struct SweptArgs {
    const double* __restrict__ bin;  // [ITS][nv][nx][ny], index 0 = oldest level
    double* __restrict__ bout;       // same layout, levels of the next half-cycle
    double* __restrict__ xface;      // [nb][Hmax-1][2][nv][2*OPS][ny]
    double* __restrict__ yface;      // [nb*nseg][2][Hmax-1][nv][Bx][2*OPS]
    double* __restrict__ frames;     // optional [nframes][nv][nx][ny]
    long long frame_cap;             // number of frame slots
    int frame_every;                 // store every k-th full step
    int nx, ny, nv, bx, hx;
    int H;        // levels in this half-cycle (<= Hmax)
    int Hmax;     // levels the face buffers were sized for
    int nb;       // bands (nx / bx)
    int nseg, wy, nchunks;
    // column segment s spans [seg_start(s), seg_start(s+1)): boundaries at
    // multiples of seg_unit, spread as evenly as seg_units allows
    int seg_unit, seg_units;
    int off;      // first row of prism band 0 (prism bands: off + i*bx)
    int its;
    // 1: the seams read each level's faces from HBM when they reach it
    // instead of staging all of them in shared memory first (seam_direct)
    int seam_direct;
    long long L0;  // global level index of this half-cycle's level 0
    int gts_base;  // the step function sees globalTimeStep = gts_base + level
    EqParams p;
};

__device__ __forceinline__ int wrap(int v, int n)
{
    v %= n;
    return v < 0 ? v + n : v;
}

// Column of the x-face buffers that holds grid column g at level m: faces are
// stored shifted by m columns, so that the register streams, whose chunks
// slide one column left per level, write and read every level's faces at the
// chunk's level-0 columns (16-byte aligned pairs).  All kernels use it.
__device__ __forceinline__ int xface_col(int g, int m, int ny)
{
    const int c = g + m;
    return c >= ny ? c - ny : c;
}

__device__ __forceinline__ int seg_start(const SweptArgs& a, int s)
{
    return a.seg_unit * (int)(((long long)s * a.seg_units) / a.nseg);
}

// Unit i = band * nseg + segment: its band, columns [s0, s1) and the unit
// whose right edge meets its left edge (for the seam at s0).
struct SegGeom {
    int band, s0, s1, left;
};
__device__ __forceinline__ SegGeom seg_geom(const SweptArgs& a, int i)
{
    const int band = i / a.nseg, seg = i % a.nseg;
    return SegGeom{band, seg_start(a, seg), seg_start(a, seg + 1),
                   band * a.nseg + (seg + a.nseg - 1) % a.nseg};
}

// Global -> shared copies that complete asynchronously (cp.async; one
// commit group per batch, wait_group<N> waits until at most N groups of this
// thread are still in flight).  16 bytes bypass L1 (.cg); 4 and 8 go through
// it (.ca, the only form for those sizes).
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}

__device__ __forceinline__ void cp_async4(void* smem, const void* gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}

// one element of T (8 bytes for double, 4 for float)
template <class T>
__device__ __forceinline__ void cp_async_elem(T* smem, const T* gmem)
{
    if constexpr (sizeof(T) == 8)
        cp_async8(smem, gmem);
    else
        cp_async4(smem, gmem);
}

__device__ __forceinline__ void cp_async_commit()
{
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}

template <int N>
__device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Seam kernels stage the faces of every level of the half-cycle in shared
// memory before the first level (the stream kernels wrote them all before
// the seam launch), so no level waits on a global load.  Per level m the
// staged y-faces are nv*nr*2OPS values per side (nr: the level's rows), the
// gap's staged x-face rows nv*2*2OPS*(2*OPS*m + 2*2OPS) values.
__host__ __device__ inline int seam_rows(bool gap, int bx, int ops, int m)
{
    return gap ? 2 * ops * m : bx - 2 * ops * m;
}
// staged y-face values of levels 1 .. m-1 (both sides)
__host__ __device__ inline int seam_yoff(bool gap, int bx, int ops, int nv, int m)
{
    // sum over levels 1..m-1 of 2 * nv * rows * 2OPS
    const int rows = gap ? ops * m * (m - 1) : (m - 1) * bx - ops * m * (m - 1);
    return 2 * nv * 2 * ops * rows;
}
// staged x-face values of levels 1 .. m-1 (gap only)
__host__ __device__ inline int seam_xoff(int ops, int nv, int m)
{
    // sum over levels 1..m-1 of nv * 2 * 2OPS * (2*OPS*m' + 2*2OPS)
    return nv * 4 * ops * (ops * m * (m - 1) + 4 * ops * (m - 1));
}
// Shared memory of one seam CTA in elements: nslot tile slots (its+1 for the
// built-in equations' ring, hmax+2 for step hooks' linear slots), then the
// staged faces of levels 1 .. hmax-1.
__host__ __device__ inline size_t seam_smem_elems(bool gap, int bx, int ops, int nv, int its,
                                                  int hmax, int nslot = 0)
{
    if (nslot == 0) nslot = its + 1;
    const size_t slots = (size_t)nslot * nv * bx * (2 * ops * (hmax + 1));
    return slots + seam_yoff(gap, bx, ops, nv, hmax) + (gap ? seam_xoff(ops, nv, hmax) : 0);
}

// Whether the seams skip the staging: where the staged faces would leave
// two or fewer seam CTAs per SM and the bare tile slots fit more (large
// Euler tiles; heat tiles keep seven with staging).
__host__ __device__ inline bool seam_direct(int bx, int ops, int nv, int its, int hmax,
                                            size_t esize, int nslot = 0)
{
    if (nslot == 0) nslot = its + 1;
    const size_t cap = 227 * 1024;
    const size_t ys = seam_smem_elems(false, bx, ops, nv, its, hmax, nslot);
    const size_t gs = seam_smem_elems(true, bx, ops, nv, its, hmax, nslot);
    const size_t staged = esize * (ys > gs ? ys : gs);
    const size_t bare = esize * (size_t)nslot * nv * bx * (2 * ops * (hmax + 1));
    return cap / staged <= 2 && cap / bare > cap / staged;
}

// Frame slot for global level L, or -1.
__device__ __forceinline__ long long frame_slot(const SweptArgs& a, long long L)
{
    if (!a.frames || L <= 0 || (L % a.its) != 0) return -1;
    long long step = L / a.its;
    if (step % a.frame_every) return -1;
    long long s = step / a.frame_every - 1;
    return s < a.frame_cap ? s : -1;
}

// Shared-memory slot of level L in a stream or seam tile.  The built-in
// equations use a ring of ITS+1 slots.  User step hooks address the previous
// and next level as idx - TIMES and idx + TIMES (pysweep/equations/heat.cu:
// 35-41), which needs the three levels at equal strides: LINEAR keeps level L
// in slot L+1 (levels -1 and 0 first), i.e. Hmax+2 slots per tile.
template <bool LINEAR, int ITS>
__host__ __device__ __forceinline__ int slot_index(int L)
{
    if (LINEAR) return L + 1;
    const int r = L % (ITS + 1);
    return r < 0 ? r + ITS + 1 : r;
}
template <bool LINEAR, int ITS>
__host__ __device__ __forceinline__ int slot_count(int hmax)
{
    return LINEAR ? hmax + 2 : ITS + 1;
}

// Equations whose functor evaluates a whole stream level at once (faces
// shared between cells): Eq::kFaceLevel and Eq::level<NT>.
template <class Eq, class = void>
struct FaceLevel {
    static constexpr bool value = false;
};
template <class Eq>
struct FaceLevel<Eq, decltype((void)Eq::kFaceLevel)> {
    static constexpr bool value = Eq::kFaceLevel;
};

// ---------------------------------------------------------------- stream ----
// One CTA = one (band, segment) block.  GAP = false: prism (UpPyramid);
// GAP = true: gap (XBridge) centred on the band's upper boundary row.
template <class Eq, int ITS, int W, bool GAP, int NT, bool LINEAR = false>
__device__ __forceinline__ void stream_body(const SweptArgs& a, const int unit, double* sm)
{
    constexpr int OPS = Eq::OPS, O2 = 2 * OPS, RS = W + O2;
    constexpr int RG = NT / W;  // row groups
    const int nv = a.nv, BX = a.bx, H = a.H, hx = a.hx, nx = a.nx, ny = a.ny;
    const int SL = nv * BX * RS;  // one level slot
    const int CS = nv * BX * O2;  // one carry
    double* slot = sm;
    double* carry = sm + slot_count<LINEAR, ITS>(a.Hmax) * SL;
    auto slot_at = [&](int L) { return slot + slot_index<LINEAR, ITS>(L) * SL; };
    const int band = unit / a.nseg, seg = unit % a.nseg;
    const int r0 = GAP ? (a.off + band * BX - hx) : (a.off + band * BX);
    const int r0w = wrap(r0, nx);
    const int s0 = seg * a.wy;
    const int tid = threadIdx.x;
    const int tk = tid % W, tr = tid / W;
    const int HF = a.Hmax - 1;
    Nbr nb;
    nb.vs = BX * RS;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        nb.x[k] = (k - 2) * RS;
        nb.y[k] = k - 2;
    }

    for (int c = 0; c < a.nchunks; ++c) {
        const int cw = s0 + c * W;
        const bool first = (c == 0), last = (c == a.nchunks - 1);
        const int Wc = last ? a.wy - c * W : W;  // the last chunk may be narrower
        const int RC = Wc + O2;                  // columns of this chunk's level slots
        // ---- level 0 and level -1 from the base --------------------------
        {
            const int lo0 = GAP ? hx - O2 : 0, hi0 = GAP ? hx + O2 : BX;
            double* s0p = slot_at(0);  // slot of level 0
            const double* b0 = a.bin + (size_t)(ITS - 1) * nv * nx * ny;
            const int n0 = nv * (hi0 - lo0) * RC;
            // level 0 (and level -1) arrive by cp.async: every copy of a
            // thread is in flight at once
            for (int e = tid; e < n0; e += NT) {
                const int k = e % RC, t = e / RC;
                const int i = lo0 + t % (hi0 - lo0), v = t / (hi0 - lo0);
                const int g = wrap(cw - O2 + k, ny), r = wrap(r0 + i, nx);
                cp_async8(s0p + (v * BX + i) * RS + k, b0 + ((size_t)v * nx + r) * ny + g);
            }
            if (ITS >= 2) {
                const int lo1 = GAP ? hx - OPS : OPS, hi1 = GAP ? hx + OPS : BX - OPS;
                double* s1p = slot_at(-1);  // slot of level -1
                const double* b1 = a.bin + (size_t)(ITS - 2) * nv * nx * ny;
                const int n1 = nv * (hi1 - lo1) * Wc;
                for (int e = tid; e < n1; e += NT) {
                    const int k = e % Wc, t = e / Wc;
                    const int i = lo1 + t % (hi1 - lo1), v = t / (hi1 - lo1);
                    const int g = wrap(cw - OPS + k, ny), r = wrap(r0 + i, nx);
                    cp_async8(s1p + (v * BX + i) * RS + k, b1 + ((size_t)v * nx + r) * ny + g);
                }
            }
            cp_async_commit();
            cp_async_wait<0>();
        }
        __syncthreads();

        for (int m = 1; m <= H; ++m) {
            const int rlo = GAP ? hx - OPS * m : OPS * m;
            const int rhi = GAP ? hx + OPS * m : BX - OPS * m;
            const int klo = first ? O2 * (m + 1) : O2;
            double* out = slot_at(m);
            const double* cur = slot_at(m - 1);
            const double* prv = slot_at(m - 2);
            const int gts = a.gts_base + (int)(a.L0 + m);
            // gap: the prisms' rows of level m that the next level reads go
            // into level m's slot by cp.async while the level is computed
            // (rows outside the level's own, a slot no level still reads)
            if (GAP && m <= H - 1) {
                const int nrow = 2 * O2;  // top band's bottom face + bottom band's top face
                const int n = nv * nrow * Wc;
                const int bup = wrap(band - 1, a.nb), bdn = band;
                for (int e = tid; e < n; e += NT) {
                    const int k = O2 + e % Wc, t = e / Wc;
                    const int rr = t % nrow, v = t / nrow;
                    const int side = rr < O2 ? 1 : 0;      // 1 = bottom face of upper band
                    const int j = rr < O2 ? rr : rr - O2;
                    const int i = rr < O2 ? hx - OPS * m - O2 + j : hx + OPS * m + j;
                    const int bb = rr < O2 ? bup : bdn;
                    const int g = wrap(cw - OPS * m - O2 + k, ny);
                    const size_t fo =
                        ((((size_t)bb * HF + (m - 1)) * 2 + side) * nv + v) * O2 + j;
                    cp_async8(out + (v * BX + i) * RS + k, a.xface + fo * ny + xface_col(g, m, ny));
                }
                cp_async_commit();
            }
            // compute level m
            if constexpr (FaceLevel<Eq>::value) {
                // faces shared between the cells of the level (scratch after the carry)
                Eq::template level<NT>(cur, prv, out, rlo, rhi, (klo > O2 ? klo : O2) - OPS,
                                       RC - OPS, RS, BX, gts, a.p,
                                       carry + (size_t)(a.Hmax + 1) * CS, tid);
            } else {
                const int k = O2 + tk;
                if (k >= klo && k < RC) {
                    // grid column of tile column k at level m (equations that
                    // address the grid by coordinates)
                    int col = cw - OPS * m - O2 + k;
                    col += col < 0 ? ny : 0;
                    col -= col >= ny ? ny : 0;
                    for (int i = rlo + tr; i < rhi; i += RG) {
                        const int o = i * RS + k;
                        if constexpr (Coords<Eq>::value) {
                            int row = r0w + i;
                            row -= row >= nx ? nx : 0;
                            Eq::step_at(cur + o - OPS, prv + o - O2, out + o, nb, gts, nv, a.p, row,
                                        col);
                        } else {
                            Eq::step(cur + o - OPS, prv + o - O2, out + o, nb, gts, nv, a.p);
                        }
                    }
                }
            }
            // carry in (previous chunk's last 2*OPS columns of level m)
            if (!first) {
                const double* cin = carry + m * CS;
                for (int e = tid; e < CS; e += NT) {
                    const int j = e % O2, t = e / O2;  // t = v*BX + i
                    out[t * RS + j] = cin[e];
                }
            }
            // carry out of level m-1
            if (m - 1 >= 1) {
                double* cout_ = carry + (m - 1) * CS;
                for (int e = tid; e < CS; e += NT) {
                    const int j = e % O2, t = e / O2;
                    cout_[e] = cur[t * RS + W + j];
                }
            }
            if (GAP) cp_async_wait<0>();  // the face rows issued before the compute
            __syncthreads();
            // ---- outputs of level m --------------------------------------
            {
                const long long L = a.L0 + m;
                const int ncol = RC - klo;
                // x-faces (prism only)
                if (!GAP && m <= H - 1) {
                    const int n = nv * 2 * O2 * ncol;
                    for (int e = tid; e < n; e += NT) {
                        const int k = klo + e % ncol, t = e / ncol;
                        const int rr = t % (2 * O2), v = t / (2 * O2);
                        const int side = rr < O2 ? 0 : 1;  // 0 = top face, 1 = bottom face
                        const int j = rr < O2 ? rr : rr - O2;
                        const int i = side == 0 ? OPS * m + j : BX - OPS * m - O2 + j;
                        const int g = wrap(cw - OPS * m - O2 + k, ny);
                        const size_t fo =
                            ((((size_t)band * HF + (m - 1)) * 2 + side) * nv + v) * O2 + j;
                        a.xface[fo * ny + xface_col(g, m, ny)] = out[(v * BX + i) * RS + k];
                    }
                }
                // base levels of the next half-cycle and frames
                const bool tob = m > H - ITS;
                const long long fs = frame_slot(a, L);
                if (tob || fs >= 0) {
                    const int nr = rhi - rlo;
                    const int n = nv * nr * ncol;
                    double* bo = tob ? a.bout + (size_t)(m - (H - ITS) - 1) * nv * nx * ny : nullptr;
                    double* fr = fs >= 0 ? a.frames + (size_t)fs * nv * nx * ny : nullptr;
                    for (int e = tid; e < n; e += NT) {
                        const int k = klo + e % ncol, t = e / ncol;
                        const int i = rlo + t % nr, v = t / nr;
                        const int g = wrap(cw - OPS * m - O2 + k, ny), r = wrap(r0 + i, nx);
                        const double val = out[(v * BX + i) * RS + k];
                        const size_t go = ((size_t)v * nx + r) * ny + g;
                        if (bo) bo[go] = val;
                        if (fr) fr[go] = val;
                    }
                }
                // y-faces at the block's column edges
                if (m <= H - 1 && (first || last)) {
                    const int nr = rhi - rlo;
                    const int n = nv * nr * O2;
                    for (int side = 0; side < 2; ++side) {
                        if ((side == 0 && !first) || (side == 1 && !last)) continue;
                        const int kb = side == 0 ? O2 * (m + 1) : Wc;
                        double* yf = a.yface +
                                     ((((size_t)unit * 2 + side) * HF + (m - 1)) * nv) * BX * O2;
                        for (int e = tid; e < n; e += NT) {
                            const int j = e % O2, t = e / O2;
                            const int i = rlo + t % nr, v = t / nr;
                            yf[(v * BX + i) * O2 + j] = out[(v * BX + i) * RS + kb + j];
                        }
                    }
                }
            }
        }
        // carry out of level H, then free the slots for the next chunk
        if (!last) {
            const double* cur = slot_at(H);
            double* cout_ = carry + H * CS;
            for (int e = tid; e < CS; e += NT) {
                const int j = e % O2, t = e / O2;
                cout_[e] = cur[t * RS + W + j];
            }
        }
        __syncthreads();
    }
}

template <class Eq, int ITS, int W, bool GAP, int NT>
__global__ void __launch_bounds__(NT) stream_kernel(SweptArgs a)
{
    extern __shared__ double sm[];
    stream_body<Eq, ITS, W, GAP, NT>(a, blockIdx.x, sm);
}

// ------------------------------------------------------------------ seam ----
// One CTA per (band, segment): the column edge at x0 = seg*wy between segment
// seg-1 (left) and seg (right).  GAP = false: YBridge; GAP = true: the
// Octahedron's down half.  Tile columns k <-> global x0 - KC + k, KC = OPS*(Hmax+1).
// ceil(log2(n)) for n >= 1
__device__ __forceinline__ int log2_ceil(int n)
{
    return n <= 1 ? 0 : 32 - __clz(n - 1);
}

// floor(log2(n)) for n >= 1, at compile time
__host__ __device__ constexpr int log2_const(int n) { return n <= 1 ? 0 : 1 + log2_const(n / 2); }

// f(r, c) for every (r, c) in [0, nr) x [0, nc), spread over NT threads:
// c from the low bits of the thread index (a power-of-two group of at least
// nc threads, at most NT), r strided by the number of groups.  Masks and
// shifts only: no division by the run-time extents.
template <int NT, class F>
__device__ __forceinline__ void for_2d(int nr, int nc, int tid, F&& f)
{
    static_assert((NT & (NT - 1)) == 0, "NT is a power of two");
    constexpr int kLogNT = log2_const(NT);
    const int lg = min(log2_ceil(nc), kLogNT);
    const int cw = 1 << lg;
    const int c0 = tid & (cw - 1), rs = NT >> lg;
    for (int c = c0; c < nc; c += cw)
        for (int r = tid >> lg; r < nr; r += rs) f(r, c);
}

template <class Eq, int ITS, bool GAP, int NT, class T = double, bool LINEAR = false>
__device__ __forceinline__ void seam_body(const SweptArgs& a, const int unit, T* sm)
{
    const T* bin = reinterpret_cast<const T*>(a.bin);
    const T* yface = reinterpret_cast<const T*>(a.yface);
    T* xface = reinterpret_cast<T*>(a.xface);
    constexpr int OPS = Eq::OPS, O2 = 2 * OPS;
    const int nv = a.nv, BX = a.bx, H = a.H, hx = a.hx, nx = a.nx, ny = a.ny;
    const int KC = OPS * (a.Hmax + 1);
    const int TW = 2 * KC;
    const int SL = nv * BX * TW;
    T* slot = sm;
    auto slot_at = [&](int L) { return slot + slot_index<LINEAR, ITS>(L) * SL; };
    const SegGeom sg = seg_geom(a, unit);
    const int band = sg.band;
    const int x0 = sg.s0;
    const int r0 = GAP ? (a.off + band * BX - hx) : (a.off + band * BX);
    const int ul = sg.left;  // left stream segment
    const int ur = unit;     // right stream segment
    const int bup = wrap(band - 1, a.nb);
    const int tid = threadIdx.x;
    const int HF = a.Hmax - 1;
    // grid row of tile row i and grid column of tile column k (BX <= nx and
    // TW <= ny, so one wrap at most)
    const int rbase = wrap(r0, nx), cbase = wrap(x0 - KC, ny);
    auto grow = [&](int i) {
        const int r = rbase + i;
        return r >= nx ? r - nx : r;
    };
    auto gcol = [&](int k) {
        const int c = cbase + k;
        return c >= ny ? c - ny : c;
    };
    Nbr nb;
    nb.vs = BX * TW;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        nb.x[k] = (k - 2) * TW;
        nb.y[k] = k - 2;
    }
    // level 0 (columns [KC-2OPS, KC+2OPS)) and level -1 (columns [KC-OPS, KC+OPS))
    {
        const int lo0 = GAP ? hx - O2 : 0, hi0 = GAP ? hx + O2 : BX;
        const T* b0 = bin + (size_t)(ITS - 1) * nv * nx * ny;
        for (int v = 0; v < nv; ++v)
            for_2d<NT>(hi0 - lo0, 2 * O2, tid, [&](int r, int c) {
                const int i = lo0 + r, k = KC - O2 + c;
                cp_async_elem(slot_at(0) + (v * BX + i) * TW + k,
                              b0 + ((size_t)v * nx + grow(i)) * ny + gcol(k));
            });
        if (ITS >= 2) {
            const int lo1 = GAP ? hx - OPS : OPS, hi1 = GAP ? hx + OPS : BX - OPS;
            const T* b1 = bin + (size_t)(ITS - 2) * nv * nx * ny;
            T* s1p = slot_at(-1);
            for (int v = 0; v < nv; ++v)
                for_2d<NT>(hi1 - lo1, O2, tid, [&](int r, int c) {
                    const int i = lo1 + r, k = KC - OPS + c;
                    cp_async_elem(s1p + (v * BX + i) * TW + k,
                                  b1 + ((size_t)v * nx + grow(i)) * ny + gcol(k));
                });
        }
    }
    // faces of levels 1 .. H-1, staged: per level the y-faces
    // [side][v][row][j] (left block's right edge, then right block's left
    // edge) and, in the gap, the prisms' rows around it [v][rr][column]
    T* ystage = slot + slot_count<LINEAR, ITS>(a.Hmax) * SL;
    T* xstage = ystage + seam_yoff(GAP, BX, OPS, nv, a.Hmax);
    const bool direct = a.seam_direct != 0;
    for (int m = 1; m <= (direct ? 0 : H - 1); ++m) {
        const int rlo = GAP ? hx - OPS * m : OPS * m;
        const int nr = seam_rows(GAP, BX, OPS, m), n = nv * nr * O2;
        const T* yl = yface + ((((size_t)ul * 2 + 1) * HF + (m - 1)) * nv) * BX * O2;
        const T* yr = yface + ((((size_t)ur * 2 + 0) * HF + (m - 1)) * nv) * BX * O2;
        T* ys = ystage + seam_yoff(GAP, BX, OPS, nv, m);
        for (int v = 0; v < nv; ++v)
            for_2d<NT>(nr, O2, tid, [&](int r, int j) {
                const int e = (v * nr + r) * O2 + j;
                const int src = (v * BX + rlo + r) * O2 + j;
                cp_async_elem(ys + e, yl + src);
                cp_async_elem(ys + n + e, yr + src);
            });
        if (GAP) {
            const int clo = KC - OPS * m;
            const int nc = 2 * OPS * m + 2 * O2;
            T* xs = xstage + seam_xoff(OPS, nv, m);
            for (int v = 0; v < nv; ++v)
                for_2d<NT>(2 * O2, nc, tid, [&](int rr, int kk) {
                    const int side = rr < O2 ? 1 : 0;
                    const int j = rr < O2 ? rr : rr - O2;
                    const int bb = rr < O2 ? bup : band;
                    const size_t fo =
                        ((((size_t)bb * HF + (m - 1)) * 2 + side) * nv + v) * O2 + j;
                    cp_async_elem(xs + (v * 2 * O2 + rr) * nc + kk,
                                  xface + fo * ny + xface_col(gcol(clo - O2 + kk), m, ny));
                });
        }
    }
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
    for (int m = 1; m <= H; ++m) {
        const int rlo = GAP ? hx - OPS * m : OPS * m;
        const int rhi = GAP ? hx + OPS * m : BX - OPS * m;
        const int clo = KC - OPS * m, chi = KC + OPS * m;
        const int nr = rhi - rlo, nc = chi - clo;
        T* out = slot_at(m);
        const T* cur = slot_at(m - 1);
        const T* prv = slot_at(m - 2);
        const int gts = a.gts_base + (int)(a.L0 + m);
        // level m's faces go to cells of level m's slot that the level does
        // not compute (columns beside the bridge, rows around the gap), and
        // the slot's previous level is no longer read: unstaged, they are
        // copied by cp.async while the level is computed; staged, afterwards
        // from shared memory
        const int n = nv * nr * O2, nc2 = nc + 2 * O2;
        const T* yl = yface + ((((size_t)ul * 2 + 1) * HF + (m - 1)) * nv) * BX * O2;
        const T* yr = yface + ((((size_t)ur * 2 + 0) * HF + (m - 1)) * nv) * BX * O2;
        if (direct && m <= H - 1) {
            for (int v = 0; v < nv; ++v)
                for_2d<NT>(nr, O2, tid, [&](int r, int j) {
                    const int src = (v * BX + rlo + r) * O2 + j;
                    T* row = out + (v * BX + rlo + r) * TW;
                    cp_async_elem(row + clo - O2 + j, yl + src);
                    cp_async_elem(row + chi + j, yr + src);
                });
            if (GAP) {
                for (int v = 0; v < nv; ++v)
                    for_2d<NT>(2 * O2, nc2, tid, [&](int rr, int kk) {
                        const int j = rr < O2 ? rr : rr - O2;
                        const int i = rr < O2 ? hx - OPS * m - O2 + j : hx + OPS * m + j;
                        const int side = rr < O2 ? 1 : 0;
                        const int bb = rr < O2 ? bup : band;
                        const size_t fo =
                            ((((size_t)bb * HF + (m - 1)) * 2 + side) * nv + v) * O2 + j;
                        cp_async_elem(out + (v * BX + i) * TW + clo - O2 + kk,
                                      xface + fo * ny + xface_col(gcol(clo - O2 + kk), m, ny));
                    });
            }
            cp_async_commit();
        }
        for_2d<NT>(nr, nc, tid, [&](int r, int c) {
            const int o = (rlo + r) * TW + clo + c;
            if constexpr (Coords<Eq>::value)
                Eq::step_at(cur + o, prv + o, out + o, nb, gts, nv, a.p, grow(rlo + r),
                            gcol(clo + c));
            else
                Eq::step(cur + o, prv + o, out + o, nb, gts, nv, a.p);
        });
        if (!direct && m <= H - 1) {
            // y-faces of level m: left part from the left block's right edge,
            // right part from the right block's left edge.
            const T* ys = ystage + seam_yoff(GAP, BX, OPS, nv, m);
            for (int v = 0; v < nv; ++v)
                for_2d<NT>(nr, O2, tid, [&](int r, int j) {
                    const int e = (v * nr + r) * O2 + j;
                    T* row = out + (v * BX + rlo + r) * TW;
                    row[clo - O2 + j] = ys[e];
                    row[chi + j] = ys[n + e];
                });
            if (GAP) {
                // the prisms' rows around the gap, columns [clo-2OPS, chi+2OPS)
                const T* xs = xstage + seam_xoff(OPS, nv, m);
                for (int v = 0; v < nv; ++v)
                    for_2d<NT>(2 * O2, nc2, tid, [&](int rr, int kk) {
                        const int j = rr < O2 ? rr : rr - O2;
                        const int i = rr < O2 ? hx - OPS * m - O2 + j : hx + OPS * m + j;
                        out[(v * BX + i) * TW + clo - O2 + kk] = xs[(v * 2 * O2 + rr) * nc2 + kk];
                    });
            }
        }
        if (direct) cp_async_wait<0>();
        __syncthreads();
        // outputs of level m
        if (!GAP && m <= H - 1) {
            for (int v = 0; v < nv; ++v)
                for_2d<NT>(2 * O2, nc, tid, [&](int rr, int kk) {
                    const int side = rr < O2 ? 0 : 1;
                    const int j = rr < O2 ? rr : rr - O2;
                    const int i = side == 0 ? OPS * m + j : BX - OPS * m - O2 + j;
                    const int k = clo + kk;
                    const size_t fo =
                        ((((size_t)band * HF + (m - 1)) * 2 + side) * nv + v) * O2 + j;
                    xface[fo * ny + xface_col(gcol(k), m, ny)] = out[(v * BX + i) * TW + k];
                });
        }
        const bool tob = m > H - ITS;
        const long long fs = frame_slot(a, a.L0 + m);
        if (tob || fs >= 0) {
            T* bo = tob ? reinterpret_cast<T*>(a.bout) + (size_t)(m - (H - ITS) - 1) * nv * nx * ny
                        : nullptr;
            T* fr = fs >= 0 ? reinterpret_cast<T*>(a.frames) + (size_t)fs * nv * nx * ny : nullptr;
            for (int v = 0; v < nv; ++v)
                for_2d<NT>(nr, nc, tid, [&](int r, int kk) {
                    const int i = rlo + r, k = clo + kk;
                    const T val = out[(v * BX + i) * TW + k];
                    const size_t go = ((size_t)v * nx + grow(i)) * ny + gcol(k);
                    if (bo) bo[go] = val;
                    if (fr) fr[go] = val;
                });
        }
    }
}

template <class Eq, int ITS, bool GAP, int NT, class T = double>
__global__ void __launch_bounds__(NT) seam_kernel(SweptArgs a)
{
    extern __shared__ double sm[];
    seam_body<Eq, ITS, GAP, NT, T>(a, blockIdx.x, reinterpret_cast<T*>(sm));
}

}  // namespace psb
