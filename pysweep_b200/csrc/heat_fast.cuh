// Register-resident prism / gap streams for the heat equation, forward Euler
// (its = 1, ops = 1, one variable): the hot kernels of the swept path.
//
// Same decomposition and the same global buffers as stream_kernel in
// swept.cuh (the seam kernels there are shared), organised for registers:
//
//   * one warp = one (band, column segment) unit; a CTA holds 4 independent
//     warps;
//   * the segment is streamed in 64-column chunks; lane l holds columns
//     2l and 2l+1 of the chunk for the band's rows, in registers (a0[], a1[]);
//   * the chunk is a parallelogram: level m covers columns
//     [cw - m, cw + 64 - m), so when level m is computed from level m-1 every
//     lane takes its left neighbour's pair with one shfl_up per column, and
//     lane 0 takes the previous chunk's last two columns (the "carry") from
//     shared memory;
//   * every register index is a compile-time constant.  The prism
//     (UpPyramid) keeps level m's rows [m, BX-m) at indices [0, BX-2m): the
//     shrinking range is a prefix, updated in place in ascending order with an
//     early exit.  The gap (XBridge) keeps level m's rows [hx-m-2, hx+m)
//     (two face rows of the upper prism plus its own rows) at indices
//     [0, 2m+2) and the two face rows of the lower prism in scalar registers;
//     it is updated in place in descending order.
//
// Per cell: 8 FP64 operations (numpy's operation order, see Heat in
// equations.cuh) and one 64-bit shuffle; no shared-memory traffic except the
// carry, which is double-buffered by chunk parity (the previous chunk's carry
// is read while this chunk's is written).
#pragma once
#include "swept.cuh"

namespace psb {

__device__ __forceinline__ double heat_fe(double c, double xm, double xp, double ym, double yp,
                                          double cr)
{
    const double dxx = __dmul_rn(cr, __dadd_rn(__fma_rn(-2.0, c, xp), xm));
    const double dyy = __dmul_rn(cr, __dadd_rn(__fma_rn(-2.0, c, yp), ym));
    return __dadd_rn(__dadd_rn(dxx, dyy), c);
}

// A lane's column pair starts on an even column at even levels and on an odd
// column at odd levels (the chunk shifts one column per level); 16-byte
// vector accesses are only legal in the even case (`even` is warp-uniform).
// In the odd case the pair may straddle the periodic column boundary, so the
// second column index g1 is wrapped separately.
__device__ __forceinline__ void st_pair(double* row, int g, int g1, double x, double y, bool even)
{
    if (even) {
        *reinterpret_cast<double2*>(row + g) = make_double2(x, y);
    } else {
        row[g] = x;
        row[g1] = y;
    }
}

__device__ __forceinline__ double2 ld_pair(const double* row, int g, int g1, bool even)
{
    if (even) return *reinterpret_cast<const double2*>(row + g);
    return make_double2(row[g], row[g1]);
}

// Left neighbour's value: shfl_up for lanes 1..31, the carry for lane 0.
__device__ __forceinline__ double from_left(double v, double carry, int lane)
{
    const double t = __shfl_up_sync(0xffffffffu, v, 1);
    return lane == 0 ? carry : t;
}

constexpr int kFastWarps = 4;   // warps (units) per CTA
constexpr int kFastChunk = 64;  // columns per chunk

template <int BX>
constexpr size_t heat_fast_smem(int hmax)
{
    // per warp: two carry buffers of [hmax][BX+2 rows][2 columns]
    return sizeof(double) * (size_t)kFastWarps * 2 * hmax * (BX + 2) * 2;
}

// A new cell pair from this lane's old rows (up u0, centre c0/c1, down d0)
// and the left neighbour's values (column 1 at up / centre / down rows L1u,
// L1c, L1d; column 0 at the centre row L0c).
__device__ __forceinline__ void heat_pair(double L1u, double L1c, double L1d, double L0c,
                                          double u0, double c0, double d0, double c1, double cr,
                                          double& n0, double& n1)
{
    n0 = heat_fe(L1c, L1u, L1d, L0c, c0, cr);
    n1 = heat_fe(c0, u0, d0, L1c, c1, cr);
}

// Gap: the four prism face rows of level m at this lane's column pair
// (upper prism's bottom face rows, then lower prism's top face rows).
__device__ __forceinline__ void load_faces(const SweptArgs& a, int bup, int band, int HF, int m,
                                           int cw, int lane, double (&f)[4][2])
{
    const int ny = a.ny;
    const int gm = wrap(cw - m + 2 * lane, ny);
    const int gm1 = gm + 1 == ny ? 0 : gm + 1;
    const bool even = (m & 1) == 0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int side = q < 2 ? 1 : 0;
        const int j = q & 1;
        const int bb = q < 2 ? bup : band;
        const size_t fo = (((size_t)bb * HF + (m - 1)) * 2 + side) * 2 + j;
        const double2 v = ld_pair(a.xface + fo * ny, gm, gm1, even);
        f[q][0] = v.x;
        f[q][1] = v.y;
    }
}

// One (band, segment) unit of one warp; `carry` is the warp's own shared
// memory (two buffers of [Hmax][BX+2][2]).
template <int BX, bool GAP>
__device__ __forceinline__ void heat_fast_body(const SweptArgs& a, const int unit, double* carry)
{
    constexpr int hx = BX / 2;
    constexpr int CR = BX + 2;  // carry rows
    const int lane = threadIdx.x & 31;
    const int H = a.H, Hm = a.Hmax, nx = a.nx, ny = a.ny;
    const int band = unit / a.nseg, seg = unit % a.nseg;
    const int r0 = GAP ? (a.off + band * BX - hx) : (a.off + band * BX);
    const int s0 = seg_start(a, seg);
    // segments are whole multiples of 32 columns: 64-column chunks, the last
    // one possibly 32 wide (lanes 16..31 then hold columns past the segment)
    const int wseg = seg_start(a, seg + 1) - s0;
    const int nchunks = (wseg + kFastChunk - 1) / kFastChunk;
    const int lastw = wseg - (nchunks - 1) * kFastChunk;
    const double cr = a.p.d[0];
    const int CB = Hm * CR * 2;  // one carry buffer: [Hm][CR][2]
    const int HF = Hm - 1;
    const int bup = wrap(band - 1, a.nb);
    const int r0w = wrap(r0, nx);

    double a0[BX], a1[BX];
    double fb0a = 0.0, fb0b = 0.0, fb1a = 0.0, fb1b = 0.0;  // gap: lower prism's face rows
    for (int c = 0; c < nchunks; ++c) {
        const int cw = s0 + c * kFastChunk;
        const bool first = (c == 0), last = (c == nchunks - 1);
        const int nact = last ? lastw / 2 : 32;  // lanes holding this chunk's columns
        double* cin = carry + (c & 1) * CB;
        double* cout = carry + ((c + 1) & 1) * CB;
        // ---- level 0 ------------------------------------------------------
        {
            const double* b = a.bin;  // its = 1: the only base level
            const int g = wrap(cw + 2 * lane, ny);
            auto rowp = [&](int r) {  // band row r, wrapped
                int row = r0w + r;
                row -= row >= nx ? nx : 0;
                return b + (size_t)row * ny;
            };
            if (!GAP) {
#pragma unroll
                for (int i = 0; i < BX; ++i) {
                    const double2 v = *reinterpret_cast<const double2*>(rowp(i) + g);
                    a0[i] = v.x;
                    a1[i] = v.y;
                }
            } else {
#pragma unroll
                for (int k = 0; k < 2; ++k) {
                    const double2 v = *reinterpret_cast<const double2*>(rowp(hx - 2 + k) + g);
                    a0[k] = v.x;
                    a1[k] = v.y;
                }
                const double2 v0 = *reinterpret_cast<const double2*>(rowp(hx) + g);
                const double2 v1 = *reinterpret_cast<const double2*>(rowp(hx + 1) + g);
                fb0a = v0.x;
                fb0b = v0.y;
                fb1a = v1.x;
                fb1b = v1.y;
            }
            // carry of level 0: columns cw-2 and cw-1 of the level's rows
            const int nrow0 = GAP ? 4 : BX;
            const int rbase = GAP ? hx - 2 : 0;
            const int gl = wrap(cw - 2, ny), gl1 = wrap(cw - 1, ny);
            for (int k = lane; k < nrow0; k += 32) {
                const double* src = rowp(rbase + k);
                cin[k * 2 + 0] = src[gl];
                cin[k * 2 + 1] = src[gl1];
            }
        }
        // gap: the faces of level 1 are read while level 0 settles
        double nf[4][2];
        if (GAP && H >= 2) load_faces(a, bup, band, HF, 1, cw, lane, nf);
        __syncwarp();
        for (int m = 1; m <= H; ++m) {
            const double* cr0 = cin + (m - 1) * CR * 2;  // carry of level m-1
            const int gm = wrap(cw - m + 2 * lane, ny);  // this lane's first column at level m
            const int gm1 = gm + 1 == ny ? 0 : gm + 1;   // and its second
            const bool even = (m & 1) == 0;              // parity of gm (cw and ny are even)
            // left-seam mask: the first chunk's level m starts at column s0+m
            // (lane m); a 32-column last chunk ends at lane 15
            const bool valid = (!first || lane >= m) && lane < nact;
            int nrow;  // rows of level m held in the arrays
            double lb0a = 0.0, lb0b = 0.0, lb1a = 0.0, lb1b = 0.0;  // prism: last two rows
            double nn[4][2];  // gap: face rows of level m+1, issued now
            if (!GAP) {
                // ---- prism: level m rows [m, BX-m) at indices [0, BX-2m) ----
                // old index i <-> row m-1+i; new index i <-> row m+i
                const int count = BX - 2 * m;
                nrow = count;
                const double2 cu = *reinterpret_cast<const double2*>(cr0 + 0);
                double2 cc = *reinterpret_cast<const double2*>(cr0 + 2);
                double L1u = from_left(a1[0], cu.y, lane);
                double L1c = from_left(a1[1], cc.y, lane);
#pragma unroll
                for (int i = 0; i < BX - 2; ++i) {
                    if (i >= count) break;
                    const double2 cd = *reinterpret_cast<const double2*>(cr0 + (i + 2) * 2);
                    const double L1d = from_left(a1[i + 2], cd.y, lane);
                    const double L0c = from_left(a0[i + 1], cc.x, lane);
                    double n0, n1;
                    heat_pair(L1u, L1c, L1d, L0c, a0[i], a0[i + 1], a0[i + 2], a1[i + 1], cr, n0,
                              n1);
                    a0[i] = n0;
                    a1[i] = n1;
                    L1u = L1c;
                    L1c = L1d;
                    cc = cd;
                    lb0a = lb1a;
                    lb0b = lb1b;
                    lb1a = n0;
                    lb1b = n1;
                }
            } else {
                // ---- gap: issue the prisms' face rows of level m+1 ---------
                // (level m's rows were issued one level step earlier)
                if (m + 1 <= H - 1) load_faces(a, bup, band, HF, m + 1, cw, lane, nn);
                // ---- level m rows [hx-m, hx+m) at indices [2, 2m+2) ----------
                // old index k <-> row hx-m-1+k for k < 2m; old rows 2m, 2m+1 are
                // the scalars fb0, fb1; new index k <-> row hx-m-2+k reads old
                // rows k-2 (up), k-1 (centre), k (down).
                const int K0 = 2 * m + 1;
                nrow = 2 * m + 2;
                double2 cc = *reinterpret_cast<const double2*>(cr0 + (K0 - 1) * 2);
                const double2 cdn = *reinterpret_cast<const double2*>(cr0 + K0 * 2);
                double L1d = from_left(fb1b, cdn.y, lane);
                double L1c = from_left(fb0b, cc.y, lane);
#pragma unroll
                for (int k = BX - 1; k >= 2; --k) {
                    if (k > K0) continue;
                    const bool top1 = (k == K0), top2 = (k == K0 - 1);
                    const double u0 = a0[k - 2], u1 = a1[k - 2];
                    const double c0 = top1 ? fb0a : a0[k - 1];
                    const double c1 = top1 ? fb0b : a1[k - 1];
                    const double d0 = top1 ? fb1a : (top2 ? fb0a : a0[k]);
                    const double2 cu = *reinterpret_cast<const double2*>(cr0 + (k - 2) * 2);
                    const double L1u = from_left(u1, cu.y, lane);
                    const double L0c = from_left(c0, cc.x, lane);
                    double n0, n1;
                    heat_pair(L1u, L1c, L1d, L0c, u0, c0, d0, c1, cr, n0, n1);
                    a0[k] = n0;
                    a1[k] = n1;
                    L1d = L1c;
                    L1c = L1u;
                    cc = cu;
                }
                // the face rows of level m join: upper at indices 0, 1, lower in
                // the scalars
                if (m <= H - 1) {
                    a0[0] = nf[0][0];
                    a1[0] = nf[0][1];
                    a0[1] = nf[1][0];
                    a1[1] = nf[1][1];
                    fb0a = nf[2][0];
                    fb0b = nf[2][1];
                    fb1a = nf[3][0];
                    fb1b = nf[3][1];
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        nf[q][0] = nn[q][0];
                        nf[q][1] = nn[q][1];
                    }
                }
            }
            // ---- carry of level m for the next chunk (lane 31's columns) ----
            if (m <= H - 1 && !last) {
                double* co = cout + m * CR * 2;
#pragma unroll
                for (int i = 0; i < BX; ++i) {
                    if (i >= nrow) break;
                    if (lane == 31)
                        *reinterpret_cast<double2*>(co + i * 2) = make_double2(a0[i], a1[i]);
                }
                if (GAP && lane == 31) {
                    *reinterpret_cast<double2*>(co + nrow * 2) = make_double2(fb0a, fb0b);
                    *reinterpret_cast<double2*>(co + (nrow + 1) * 2) = make_double2(fb1a, fb1b);
                }
            }
            // ---- outputs of level m ------------------------------------------
            // computed rows: prism indices [0, nrow) (band rows m+i); gap
            // indices [2, nrow) (band rows hx-m-2+k)
            const int ibeg = GAP ? 2 : 0;
            const int rfirst = GAP ? hx - m - 2 : m;  // band row of index 0
            if (!GAP && m <= H - 1 && valid) {
                const size_t fb = ((size_t)band * HF + (m - 1)) * 2;
                st_pair(a.xface + ((fb + 0) * 2 + 0) * ny, gm, gm1, a0[0], a1[0], even);
                st_pair(a.xface + ((fb + 0) * 2 + 1) * ny, gm, gm1, a0[1], a1[1], even);
                st_pair(a.xface + ((fb + 1) * 2 + 0) * ny, gm, gm1, lb0a, lb0b, even);
                st_pair(a.xface + ((fb + 1) * 2 + 1) * ny, gm, gm1, lb1a, lb1b, even);
            }
            const long long fs = frame_slot(a, a.L0 + m);
            if (m == H || fs >= 0) {
                double* fr = fs >= 0 ? a.frames + (size_t)fs * nx * ny : nullptr;
#pragma unroll
                for (int i = 0; i < BX; ++i) {
                    if (i >= nrow) break;
                    if (i < ibeg) continue;
                    int row = r0w + rfirst + i;
                    row -= row >= nx ? nx : 0;
                    const size_t o = (size_t)row * ny;
                    if (m == H && valid) st_pair(a.bout + o, gm, gm1, a0[i], a1[i], even);
                    if (fr && valid) st_pair(fr + o, gm, gm1, a0[i], a1[i], even);
                }
            }
            // y-faces at the segment's column edges (read by the seam kernels)
            if (m <= H - 1 && (first || last)) {
#pragma unroll
                for (int side = 0; side < 2; ++side) {
                    if ((side == 0 && !first) || (side == 1 && !last)) continue;
                    const int owner = side == 0 ? m : nact - 1;
                    double* yf = a.yface + (((size_t)unit * 2 + side) * HF + (m - 1)) * BX * 2;
#pragma unroll
                    for (int i = 0; i < BX; ++i) {
                        if (i >= nrow) break;
                        if (i < ibeg) continue;
                        if (lane == owner)
                            *reinterpret_cast<double2*>(yf + (rfirst + i) * 2) =
                                make_double2(a0[i], a1[i]);
                    }
                }
            }
        }
        __syncwarp();
    }
}

template <int BX, bool GAP>
__global__ void __launch_bounds__(32 * kFastWarps, 3) heat_stream_fast(SweptArgs a)
{
    extern __shared__ double sm[];
    const int warp = threadIdx.x >> 5;
    const int unit = blockIdx.x * kFastWarps + warp;
    if (unit >= a.nb * a.nseg) return;  // whole warp leaves together
    heat_fast_body<BX, GAP>(a, unit, sm + (size_t)warp * 2 * (a.Hmax * (BX + 2) * 2));
}

}  // namespace psb
