// Register-resident y-bridge seam for heat with forward Euler (its = 1,
// ops = 1, float64): the YBridge phase (pysweep/core/pysweep.cu:99-128) of the
// register streams' decomposition, bit-identical to seam_kernel<Heat, 1,
// false> (same cells, same per-cell arithmetic, same outputs).
//
// One warp per column edge x0 of a (band, segment) unit.  Lane k holds tile
// column k <-> grid column x0 - KC + k (KC = Hmax + 1, so 2 KC <= 32 lanes at
// blocksize 32), all bs rows of the band in registers.  Level m computes rows
// [m, bs-m) at columns [KC-m, KC+m) from level m-1 at columns
// [KC-m-1, KC+m+1): its own rows sit in the lane's registers, the columns
// beside it arrive by shuffle.  The rows use the prism stream's in-place
// layout (level m's row m+i at register index i, updated in ascending order),
// so a level needs no second copy; lanes outside the level's columns compute
// values nobody reads.  After level m the four lanes just outside its columns
// take the streams' y-faces of level m (two columns per side, staged in
// shared memory by cp.async when the kernel starts), which the next level
// reads.  Compared with the shared-memory seam, no tile slots, barriers or
// per-cell index arithmetic: about 15 instructions per lane and row.
#pragma once
#include "heat_fast.cuh"

namespace psb {

constexpr int kSeamWarps = 4;  // seams (warps) per CTA

// Staged y-faces of one warp, in doubles: [side][level 1 .. Hmax-1][row][2].
template <int BX>
__host__ __device__ constexpr int yseam_warp_doubles(int hmax)
{
    return 2 * (hmax - 1) * BX * 2;
}

template <int BX>
constexpr size_t yseam_smem(int hmax)
{
    return sizeof(double) * (size_t)kSeamWarps * yseam_warp_doubles<BX>(hmax);
}

// The bottom x-face rows of level m are the last two of its `count` rows.
#define PSB_YSEAM_BOTTOM(C)                                                                \
    case C:                                                                                \
        if constexpr ((C) <= BX) {                                                         \
            f1[0] = v[(C) - 2];                                                            \
            f1[ny] = v[(C) - 1];                                                           \
        }                                                                                  \
        break;

template <int BX>
__device__ __forceinline__ void yseam_bottom(int count, const double (&v)[BX], double* f1, int ny)
{
    static_assert(BX <= 32, "cases cover blocksizes up to 32");
    switch (count) {
        PSB_YSEAM_BOTTOM(2) PSB_YSEAM_BOTTOM(4) PSB_YSEAM_BOTTOM(6) PSB_YSEAM_BOTTOM(8)
        PSB_YSEAM_BOTTOM(10) PSB_YSEAM_BOTTOM(12) PSB_YSEAM_BOTTOM(14) PSB_YSEAM_BOTTOM(16)
        PSB_YSEAM_BOTTOM(18) PSB_YSEAM_BOTTOM(20) PSB_YSEAM_BOTTOM(22) PSB_YSEAM_BOTTOM(24)
        PSB_YSEAM_BOTTOM(26) PSB_YSEAM_BOTTOM(28) PSB_YSEAM_BOTTOM(30) PSB_YSEAM_BOTTOM(32)
        default: break;
    }
}
#undef PSB_YSEAM_BOTTOM

template <int BX>
__device__ __forceinline__ void heat_yseam_body(const SweptArgs& a, const int unit, double* ys)
{
    const int lane = threadIdx.x & 31;
    const int H = a.H, Hm = a.Hmax, nx = a.nx, ny = a.ny;
    const int KC = Hm + 1;
    const int HF = Hm - 1;
    const SegGeom sg = seg_geom(a, unit);
    const int band = sg.band;
    const int r0w = wrap(a.off + band * BX, nx);
    const double cr = a.p.d[0];
    const int gc = wrap(sg.s0 - KC + lane, ny);  // this lane's grid column
    auto grow = [&](int r) {                     // grid row of band row r
        int row = r0w + r;
        row -= row >= nx ? nx : 0;
        return row;
    };
    // y-faces of levels 1 .. H-1: the left unit's right edge (side 1) and
    // this unit's left edge (side 0), [level][row][2] each, contiguous
    {
        const double* yl = a.yface + ((size_t)sg.left * 2 + 1) * HF * BX * 2;
        const double* yr = a.yface + ((size_t)unit * 2 + 0) * HF * BX * 2;
        const int npair = (H - 1) * BX;  // 16-byte pairs per side
        for (int e = lane; e < npair; e += 32) {
            cp_async16(ys + e * 2, yl + e * 2);
            cp_async16(ys + (HF * BX + e) * 2, yr + e * 2);
        }
        cp_async_commit();
    }
    // level 0 at columns KC-2 .. KC+1, every row
    double v[BX];
    const bool base_lane = lane >= KC - 2 && lane < KC + 2;
#pragma unroll
    for (int i = 0; i < BX; ++i) v[i] = base_lane ? a.bin[(size_t)grow(i) * ny + gc] : 0.0;
    cp_async_wait<0>();
    __syncwarp();
    for (int m = 1; m <= H; ++m) {
        const int count = BX - 2 * m;  // rows of level m: band rows m .. m+count-1
        // ---- level m, in place: index i <-> row m+i (old: row m-1+i) ------
#pragma unroll
        for (int i = 0; i < BX - 2; ++i) {
            if (i >= count) break;
            const double c = v[i + 1];
            const double ym = __shfl_up_sync(0xffffffffu, c, 1);
            const double yp = __shfl_down_sync(0xffffffffu, c, 1);
            v[i] = heat_fe(c, v[i], v[i + 2], ym, yp, cr);
        }
        const bool mine = lane >= KC - m && lane < KC + m;  // the level's own columns
        // ---- x-faces of level m (rows m, m+1 and bs-m-2, bs-m-1) --------------
        if (m <= H - 1 && mine) {
            const size_t fb = ((size_t)band * HF + (m - 1)) * 2;
            const int xc = xface_col(gc, m, ny);
            double* f0 = a.xface + ((fb + 0) * 2) * ny + xc;
            double* f1 = a.xface + ((fb + 1) * 2) * ny + xc;
            f0[0] = v[0];
            f0[ny] = v[1];
            yseam_bottom<BX>(count, v, f1, ny);
        }
        // ---- base level of the next half-cycle and frames ---------------------
        const long long fs = frame_slot(a, a.L0 + m);
        if ((m == H || fs >= 0) && mine) {
            double* fr = fs >= 0 ? a.frames + (size_t)fs * nx * ny : nullptr;
#pragma unroll
            for (int i = 0; i < BX; ++i) {
                if (i >= count) break;
                const size_t o = (size_t)grow(m + i) * ny + gc;
                if (m == H) a.bout[o] = v[i];
                if (fr) fr[o] = v[i];
            }
        }
        // ---- the streams' y-faces of level m join beside the level's columns --
        if (m <= H - 1) {
            const int side = lane < KC ? 0 : 1;               // 0: left unit, 1: this unit
            const int j = side == 0 ? lane - (KC - m - 2) : lane - (KC + m);
            const bool face = j >= 0 && j < 2;
            const double* src = ys + ((side * HF + (m - 1)) * BX + m) * 2 + (j & 1);
#pragma unroll
            for (int i = 0; i < BX; ++i) {
                if (i >= count) break;
                if (face) v[i] = src[i * 2];
            }
        }
    }
}

template <int BX>
__global__ void __launch_bounds__(32 * kSeamWarps) heat_yseam_fast(SweptArgs a)
{
    extern __shared__ double sm[];
    const int warp = threadIdx.x >> 5;
    const int unit = blockIdx.x * kSeamWarps + warp;
    if (unit >= a.nb * a.nseg) return;  // whole warp leaves together
    heat_yseam_body<BX>(a, unit, sm + (size_t)warp * yseam_warp_doubles<BX>(a.Hmax));
}

// ---------------------------------------------------------------- octahedron
// The Octahedron's down half (pysweep/core/pysweep.cu:164-217) at a column
// edge of the gap band: level m computes rows [hx-m, hx+m) at columns
// [KC-m, KC+m) (the shared-memory seam_kernel<Heat, 1, true>'s cells and
// arithmetic).  Registers hold the gap stream's layout: before level m, index
// k <-> row hx-m-1+k for k in [0, 2m+2) (indices 0, 1 and 2m, 2m+1: the
// prisms' face rows of level m-1, x-faces); level m is computed in place from
// index 2m+1 down to 2 (new index k <-> row hx-m-2+k reads old k-2, k-1, k),
// entered at its first row through a switch.  After level m every lane of
// columns [KC-m-2, KC+m+2) takes the four x-face rows of level m (loaded while
// the level was computed; the lower two join at the next level's entry, on
// the path of the switch case that enters it, as in the gap stream) and the
// four lanes beside the level's columns take the gap streams' y-faces of
// level m (staged in shared memory).

template <int BX>
__device__ __forceinline__ void heat_oseam_body(const SweptArgs& a, const int unit, double* ys)
{
    constexpr int hx = BX / 2;
    const int lane = threadIdx.x & 31;
    const int H = a.H, Hm = a.Hmax, nx = a.nx, ny = a.ny;
    const int KC = Hm + 1;
    const int HF = Hm - 1;
    const SegGeom sg = seg_geom(a, unit);
    const int band = sg.band;
    const int bup = wrap(band - 1, a.nb);
    const int r0w = wrap(a.off + band * BX - hx, nx);  // gap band row 0
    const double cr = a.p.d[0];
    const int gc = wrap(sg.s0 - KC + lane, ny);  // this lane's grid column
    auto grow = [&](int r) {
        int row = r0w + r;
        row -= row >= nx ? nx : 0;
        return row;
    };
    {
        const double* yl = a.yface + ((size_t)sg.left * 2 + 1) * HF * BX * 2;
        const double* yr = a.yface + ((size_t)unit * 2 + 0) * HF * BX * 2;
        const int npair = (H - 1) * BX;
        for (int e = lane; e < npair; e += 32) {
            cp_async16(ys + e * 2, yl + e * 2);
            cp_async16(ys + (HF * BX + e) * 2, yr + e * 2);
        }
        cp_async_commit();
    }
    // level 0: rows hx-2 .. hx+1 at columns KC-2 .. KC+1 (indices 0 .. 3)
    double v[BX];
#pragma unroll
    for (int i = 0; i < BX; ++i) v[i] = 0.0;
    if (lane >= KC - 2 && lane < KC + 2) {
#pragma unroll
        for (int i = 0; i < 4; ++i) v[i] = a.bin[(size_t)grow(hx - 2 + i) * ny + gc];
    }
    cp_async_wait<0>();
    __syncwarp();
    // x-face rows of level m at this lane's column: upper prism's bottom rows
    // (j = 0, 1), lower prism's top rows
    auto xrow = [&](int bb, int side, int j, int m) {
        const size_t fo = (((size_t)bb * HF + (m - 1)) * 2 + side) * 2 + j;
        return a.xface + fo * ny + xface_col(gc, m, ny);
    };
    double f0 = 0.0, f1 = 0.0, f2 = 0.0, f3 = 0.0;
    double p2 = 0.0, p3 = 0.0;  // lower face rows of the previous level
    for (int m = 1; m <= H; ++m) {
        // this level's x-faces, placed after the level (they are the next
        // level's rows); loaded now so the level's arithmetic covers them
        if (m <= H - 1) {
            f0 = *xrow(bup, 1, 0, m);
            f1 = *xrow(bup, 1, 1, m);
            f2 = *xrow(band, 0, 0, m);
            f3 = *xrow(band, 0, 1, m);
        }
        // ---- level m, in place from index 2m+1 down to 2 ---------------------
        // (entering level m places the lower face rows of level m-1 at
        // indices 2m, 2m+1; at m = 1 they are the base rows of level 0)
#define PSB_OSEAM_ENTRY(M)                                                                 \
    case M:                                                                                \
        if constexpr ((M) >= 2 && 2 * (M) + 1 < BX) {                                      \
            v[2 * (M)] = p2;                                                               \
            v[2 * (M) + 1] = p3;                                                           \
        }                                                                                  \
        goto orow_##M;
#define PSB_OSEAM_ROW(K)                                                                   \
    if constexpr ((K) >= 2 && (K) < BX) {                                                  \
        const double c = v[(K) - 1];                                                       \
        const double ym = __shfl_up_sync(0xffffffffu, c, 1);                               \
        const double yp = __shfl_down_sync(0xffffffffu, c, 1);                             \
        v[K] = heat_fe(c, v[(K) - 2], v[K], ym, yp, cr);                                   \
    }
        switch (m) {
            PSB_OSEAM_ENTRY(15) PSB_OSEAM_ENTRY(14) PSB_OSEAM_ENTRY(13) PSB_OSEAM_ENTRY(12) PSB_OSEAM_ENTRY(11)
            PSB_OSEAM_ENTRY(10) PSB_OSEAM_ENTRY(9) PSB_OSEAM_ENTRY(8) PSB_OSEAM_ENTRY(7)
            PSB_OSEAM_ENTRY(6) PSB_OSEAM_ENTRY(5) PSB_OSEAM_ENTRY(4) PSB_OSEAM_ENTRY(3)
            PSB_OSEAM_ENTRY(2) PSB_OSEAM_ENTRY(1)
            default: goto orow_end;
        }
        // level m enters at index 2m+1 (label orow_m) and falls through to 2
    orow_15:
        PSB_OSEAM_ROW(31) PSB_OSEAM_ROW(30)
    orow_14:
        PSB_OSEAM_ROW(29) PSB_OSEAM_ROW(28)
    orow_13:
        PSB_OSEAM_ROW(27) PSB_OSEAM_ROW(26)
    orow_12:
        PSB_OSEAM_ROW(25) PSB_OSEAM_ROW(24)
    orow_11:
        PSB_OSEAM_ROW(23) PSB_OSEAM_ROW(22)
    orow_10:
        PSB_OSEAM_ROW(21) PSB_OSEAM_ROW(20)
    orow_9:
        PSB_OSEAM_ROW(19) PSB_OSEAM_ROW(18)
    orow_8:
        PSB_OSEAM_ROW(17) PSB_OSEAM_ROW(16)
    orow_7:
        PSB_OSEAM_ROW(15) PSB_OSEAM_ROW(14)
    orow_6:
        PSB_OSEAM_ROW(13) PSB_OSEAM_ROW(12)
    orow_5:
        PSB_OSEAM_ROW(11) PSB_OSEAM_ROW(10)
    orow_4:
        PSB_OSEAM_ROW(9) PSB_OSEAM_ROW(8)
    orow_3:
        PSB_OSEAM_ROW(7) PSB_OSEAM_ROW(6)
    orow_2:
        PSB_OSEAM_ROW(5) PSB_OSEAM_ROW(4)
    orow_1:
        PSB_OSEAM_ROW(3) PSB_OSEAM_ROW(2)
    orow_end:;
#undef PSB_OSEAM_ENTRY
#undef PSB_OSEAM_ROW
        const bool mine = lane >= KC - m && lane < KC + m;
        // ---- base level of the next half-cycle and frames (indices [2, 2m+2):
        // rows hx-m .. hx+m-1) ------------------------------------------------
        const long long fs = frame_slot(a, a.L0 + m);
        if ((m == H || fs >= 0) && mine) {
            double* fr = fs >= 0 ? a.frames + (size_t)fs * nx * ny : nullptr;
#pragma unroll
            for (int k = 2; k < BX; ++k) {
                if (k >= 2 * m + 2) break;
                const size_t o = (size_t)grow(hx - m - 2 + k) * ny + gc;
                if (m == H) a.bout[o] = v[k];
                if (fr) fr[o] = v[k];
            }
        }
        if (m <= H - 1) {
            // the gap streams' y-faces of level m beside the level's columns
            const int side = lane < KC ? 0 : 1;
            const int j = side == 0 ? lane - (KC - m - 2) : lane - (KC + m);
            const bool face = j >= 0 && j < 2;
            const double* src = ys + ((side * HF + (m - 1)) * BX + hx - m) * 2 + (j & 1);
#pragma unroll
            for (int k = 2; k < BX; ++k) {
                if (k >= 2 * m + 2) break;
                if (face) v[k] = src[(k - 2) * 2];
            }
            // the prisms' face rows of level m: indices 0, 1 now, 2m+2 and
            // 2m+3 on entering the next level
            v[0] = f0;
            v[1] = f1;
            p2 = f2;
            p3 = f3;
        }
    }
}

template <int BX>
__global__ void __launch_bounds__(32 * kSeamWarps) heat_oseam_fast(SweptArgs a)
{
    extern __shared__ double sm[];
    const int warp = threadIdx.x >> 5;
    const int unit = blockIdx.x * kSeamWarps + warp;
    if (unit >= a.nb * a.nseg) return;  // whole warp leaves together
    heat_oseam_body<BX>(a, unit, sm + (size_t)warp * yseam_warp_doubles<BX>(a.Hmax));
}

}  // namespace psb
