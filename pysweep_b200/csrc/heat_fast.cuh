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
//     early exit.  The gap (XBridge) keeps level m-1's rows [hx-m-1, hx+m+1)
//     (two face rows of the upper prism, its own rows, two face rows of the
//     lower prism) at indices [0, 2m+2) and updates them in place in
//     descending order, two rows at a time, entering at the level's first
//     row pair through a switch (Duff's device).  Each row pair computes its
//     left neighbours from the arrays and the carry, so no value travels from
//     one pair to the next and the entry points cost no register moves.
//
// Per cell: 8 FP64 operations (numpy's operation order, see Heat in
// equations.cuh) and one (prism) or two (gap) 64-bit shuffles.  Shared memory
// holds the carry, double-buffered by chunk parity (the previous chunk's carry
// is read while this chunk's is written) and packed by level (level j keeps
// the rows it has), and, in the gap, a ring of the prisms' face rows: the face rows of
// level m are copied with cp.async kFaceDepth levels before they are needed,
// which hides the latency of the x-face reads.  The x-faces are stored at the
// chunk's level-0 columns (xface_col in swept.cuh), so every face access is
// one aligned 16-byte pair per lane.
//
// VAR 1 and 2 are the same streams with a courant number per cell (the
// differentiable solve's forward step and its adjoint in mu = C .* lambda,
// HeatVar and HeatVarAdjMu in equations.cuh): each row's per-cell operands
// arrive through a ring in shared memory (var_issue / var_next).
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

// Storage type of the fields.  double; or float, every level evaluated in
// double and rounded to float (the reference's float32 runs: its courant is a
// float64 scalar, so numpy computes each level in float64 and rounds it when
// it is stored).  Registers, carry and arithmetic are double in both cases.
template <class T>
struct Pair2;
template <>
struct Pair2<double> {
    using type = double2;
};
template <>
struct Pair2<float> {
    using type = float2;
};

template <class T>
__device__ __forceinline__ double to_level(double x)
{
    return x;
}
template <>
__device__ __forceinline__ double to_level<float>(double x)
{
    return (double)__double2float_rn(x);
}

template <class T>
__device__ __forceinline__ typename Pair2<T>::type pair2(double x, double y);
template <>
__device__ __forceinline__ double2 pair2<double>(double x, double y)
{
    return make_double2(x, y);
}
template <>
__device__ __forceinline__ float2 pair2<float>(double x, double y)
{
    return make_float2((float)x, (float)y);  // exact: x, y already carry float precision
}

template <class P>
__device__ __forceinline__ double2 widen(P v)
{
    return make_double2((double)v.x, (double)v.y);
}

// A lane's column pair starts on an even column at even levels and on an odd
// column at odd levels (the chunk shifts one column per level); 16-byte
// vector stores are only legal in the even case (`even` is warp-uniform).
// In the odd case the pair may straddle the periodic column boundary, so the
// second column index g1 is wrapped separately.
template <class T>
__device__ __forceinline__ void st_pair(T* row, int g, int g1, double x, double y, bool even)
{
    if (even) {
        *reinterpret_cast<typename Pair2<T>::type*>(row + g) = pair2<T>(x, y);
    } else {
        row[g] = (T)x;
        row[g1] = (T)y;
    }
}

// Left neighbour's value: shfl_up for lanes 1..31, the carry for lane 0.
__device__ __forceinline__ double from_left(double v, double carry, int lane)
{
    const double t = __shfl_up_sync(0xffffffffu, v, 1);
    return lane == 0 ? carry : t;
}

constexpr int kFastWarps = 4;   // warps (units) per CTA
// CTAs per SM the register cap allows.  Bands of 32 rows: three for heat (168
// registers), two for the per-cell courant variants, whose extra operands
// would spill at 168.  Bands of 16 rows hold half the values: four (128).
__host__ __device__ constexpr int fast_ctas_per_sm(int bx, int var)
{
    return bx <= 16 ? 4 : (var == 0 ? 3 : 2);
}
template <int BX, int VAR>
constexpr int kFastCtasPerSm = fast_ctas_per_sm(BX, VAR);
constexpr int kFastChunk = 64;  // columns per chunk
constexpr int kFaceDepth = 3;   // gap: levels of face rows in flight ahead of use
constexpr int kFaceSlots = kFaceDepth + 1;

// Carry rows kept for levels 0 .. m-1 (the carry of level j holds the rows
// the level has: BX - 2j for the prism, 2j + 4 for the gap), i.e. the offset
// of level m's carry in the packed buffer.
template <int BX, bool GAP>
__host__ __device__ constexpr int carry_rows(int m)
{
    return GAP ? m * (m + 3) : m * BX - m * (m - 1);
}

// Shared memory of one warp, in doubles: two packed carry buffers (chunk
// parity) and the gap's ring of face rows ([slot][4 rows][32 lanes][2]).
template <int BX>
__host__ __device__ constexpr int heat_fast_warp_doubles(int hmax)
{
    return 2 * 2 * (carry_rows<BX, false>(hmax) > carry_rows<BX, true>(hmax)
                        ? carry_rows<BX, false>(hmax)
                        : carry_rows<BX, true>(hmax)) +
           kFaceSlots * 4 * 32 * 2;
}

template <int BX>
constexpr size_t heat_fast_smem(int hmax)
{
    return sizeof(double) * (size_t)kFastWarps * heat_fast_warp_doubles<BX>(hmax);
}

// Per-cell courant variants (VAR > 0): after the warp's carry buffers and face
// ring, a ring of kVarSlots rows of per-cell operands ([field][lane]: the
// courant numbers of the lane's two cells; for VAR 2 also the recomputed
// Laplacians and the sums), copied by cp.async kVarAhead rows before use.
constexpr int kVarSlots = 4;
constexpr int kVarAhead = kVarSlots - 1;
template <int VAR>
__host__ __device__ constexpr int var_fields()
{
    return VAR == 2 ? 6 : (VAR == 1 ? 2 : 0);
}
template <int BX, int VAR>
__host__ __device__ constexpr int heat_fast_warp_doubles_v(int hmax)
{
    return heat_fast_warp_doubles<BX>(hmax) + kVarSlots * var_fields<VAR>() * 32;
}
template <int BX, int VAR>
constexpr size_t heat_fast_smem_v(int hmax)
{
    return sizeof(double) * (size_t)kFastWarps * heat_fast_warp_doubles_v<BX, VAR>(hmax);
}

// one pair of T (16 bytes for double, 8 for float)
template <class T>
__device__ __forceinline__ void cp_async_pair(T* smem, const T* gmem)
{
    if constexpr (sizeof(T) == 8)
        cp_async16(smem, gmem);
    else
        cp_async8(smem, gmem);
}

// A new cell pair from this lane's old rows (up u0, centre c0/c1, down d0)
// and the left neighbour's values (column 1 at up / centre / down rows L1u,
// L1c, L1d; column 0 at the centre row L0c).
// The results are rounded to the storage precision of T.
template <class T = double>
__device__ __forceinline__ void heat_pair(double L1u, double L1c, double L1d, double L0c,
                                          double u0, double c0, double d0, double c1, double cr,
                                          double& n0, double& n1)
{
    n0 = to_level<T>(heat_fe(L1c, L1u, L1d, L0c, c0, cr));
    n1 = to_level<T>(heat_fe(c0, u0, d0, L1c, c1, cr));
}

// Per-cell courant numbers (heat with a variable diffusivity, VAR > 0): the
// courant field, this level's slab of the recomputed Laplacians (VAR 1: stored
// when set; VAR 2: read) and the adjoint's accumulated sum (VAR 2).
struct VarFields {
    const double* C;
    double* lu;
    double* g;
};

// The per-cell operands of one new row at this lane's two columns.
struct VarPre {
    double c0, c1, l0, l1, g0, g1;
};

// Start copying row `row`'s operands at the lane's columns gm, gm1 into one
// ring slot (8-byte cp.async: the columns of odd levels are not 16-byte
// aligned).  A sum is read here and written by this lane alone within the
// level (other lanes' writes of the level before precede the level's first
// copy, behind a __syncwarp).
template <int VAR>
__device__ __forceinline__ void var_issue(const VarFields& vf, double* slot, int row, int ny,
                                          int gm, int gm1, int lane)
{
    const size_t o = (size_t)row * ny;
    cp_async8(slot + 0 * 32 + lane, vf.C + o + gm);
    cp_async8(slot + 1 * 32 + lane, vf.C + o + gm1);
    if constexpr (VAR == 2) {
        cp_async8(slot + 2 * 32 + lane, vf.lu + o + gm);
        cp_async8(slot + 3 * 32 + lane, vf.lu + o + gm1);
        cp_async8(slot + 4 * 32 + lane, vf.g + o + gm);
        cp_async8(slot + 5 * 32 + lane, vf.g + o + gm1);
    }
}

template <int VAR>
__device__ __forceinline__ VarPre var_read(const double* slot, int lane)
{
    VarPre p{};
    p.c0 = slot[0 * 32 + lane];
    p.c1 = slot[1 * 32 + lane];
    if constexpr (VAR == 2) {
        p.l0 = slot[2 * 32 + lane];
        p.l1 = slot[3 * 32 + lane];
        p.g0 = slot[4 * 32 + lane];
        p.g1 = slot[5 * 32 + lane];
    }
    return p;
}

// Ring position q of a level (the q-th row the level computes): wait until
// its copy has landed, read it, and start the copy of position q + kVarAhead
// (row `rnext`, if the level has it) into the slot read one position ago.
template <int VAR>
__device__ __forceinline__ VarPre var_next(const VarFields& vf, double* ring, int q, bool more,
                                           int rnext, int ny, int gm, int gm1, int lane)
{
    constexpr int F = var_fields<VAR>() * 32;
    cp_async_wait<kVarAhead - 1>();
    const VarPre p = var_read<VAR>(ring + (q % kVarSlots) * F, lane);
    if (more) var_issue<VAR>(vf, ring + ((q + kVarAhead) % kVarSlots) * F, rnext, ny, gm, gm1, lane);
    cp_async_commit();
    return p;
}

// heat_pair with the courant number of each cell (p.c0, p.c1); VAR 1 also
// stores each old level's Laplacian (dxx + dyy before the courant factor, the
// order of HeatVar::step_at) at grid row `row`, VAR 2 adds the old centre
// times the recomputed Laplacian to the sum (HeatVarAdjMu::step_at).  Stores
// only where `valid` (the lane's cells belong to this stream).
template <int VAR>
__device__ __forceinline__ void heat_pair_var(double L1u, double L1c, double L1d, double L0c,
                                              double u0, double c0, double d0, double c1,
                                              const VarPre& p, const VarFields& vf, int row,
                                              int ny, int gm, int gm1, bool valid, double& n0,
                                              double& n1)
{
    const size_t o = (size_t)row * ny;
    const double g0 = p.g0, g1 = p.g1;
    const double rx0 = __dadd_rn(__fma_rn(-2.0, L1c, L1d), L1u);
    const double ry0 = __dadd_rn(__fma_rn(-2.0, L1c, c0), L0c);
    const double rx1 = __dadd_rn(__fma_rn(-2.0, c0, d0), u0);
    const double ry1 = __dadd_rn(__fma_rn(-2.0, c0, c1), L1c);
    n0 = __dadd_rn(__dadd_rn(__dmul_rn(p.c0, rx0), __dmul_rn(p.c0, ry0)), L1c);
    n1 = __dadd_rn(__dadd_rn(__dmul_rn(p.c1, rx1), __dmul_rn(p.c1, ry1)), c0);
    if constexpr (VAR == 1) {
        if (vf.lu && valid) {
            vf.lu[o + gm] = __dadd_rn(rx0, ry0);
            vf.lu[o + gm1] = __dadd_rn(rx1, ry1);
        }
    } else if constexpr (VAR == 2) {
        if (valid) {
            vf.g[o + gm] = __fma_rn(L1c, p.l0, g0);
            vf.g[o + gm1] = __fma_rn(c0, p.l1, g1);
        }
    }
}

// Grid row of new row index k of the gap (row0: the grid row of index 0).
__device__ __forceinline__ int gap_grid_row(int row0, int k, int nx)
{
    const int r = row0 + k;
    return r >= nx ? r - nx : r;
}

// Gap: start the copy of the four prism face rows of level m at this lane's
// column pair (upper prism's bottom face rows, then lower prism's top face
// rows) into one ring slot; gcol is the chunk's level-0 column of the lane.
template <class T>
__device__ __forceinline__ void issue_faces(const SweptArgs& a, int bup, int band, int HF, int m,
                                            int gcol, int lane, T* slot)
{
    const T* xface = reinterpret_cast<const T*>(a.xface);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int side = q < 2 ? 1 : 0;
        const int j = q & 1;
        const int bb = q < 2 ? bup : band;
        const size_t fo = (((size_t)bb * HF + (m - 1)) * 2 + side) * 2 + j;
        cp_async_pair<T>(slot + (q * 32 + lane) * 2, xface + fo * a.ny + gcol);
    }
}

// Gap: the lower prism's two face rows of level m-1 join the arrays at
// indices K-1 and K (K = 2m+1, the level's first pair), on the level's entry
// path into the pairs: the write has constant register indices and sits on a
// path of its own, so no other path has to merge it (a switch after the
// level, joining all cases in one place, made the compiler select every
// index it could write).  `lower` points at this lane's pair of the face
// row in the ring slot of level m-1; at m = 1 the rows are the base rows
// loaded with level 0.
template <int K, int BX, class T>
__device__ __forceinline__ void gap_lower(double (&a0)[BX], double (&a1)[BX], const T* lower)
{
    if constexpr (K >= 5 && K < BX) {
        using P = typename Pair2<T>::type;
        const double2 f2 = widen(*reinterpret_cast<const P*>(lower));
        const double2 f3 = widen(*reinterpret_cast<const P*>(lower + 64));
        a0[K - 1] = f2.x;
        a1[K - 1] = f2.y;
        a0[K] = f3.x;
        a1[K] = f3.y;
    }
}

// Prism: the bottom face rows of level m are the last two of its `count`
// rows, register indices count-2 and count-1.
#define PSB_BOTTOM_CASE(C)                                                                 \
    case C:                                                                                \
        if constexpr ((C) <= BX) {                                                         \
            *reinterpret_cast<P*>(r0) = pair2<T>(a0[(C) - 2], a1[(C) - 2]);                \
            *reinterpret_cast<P*>(r1) = pair2<T>(a0[(C) - 1], a1[(C) - 1]);                \
        }                                                                                  \
        break;

template <int BX, class T>
__device__ __forceinline__ void store_bottom(int count, const double (&a0)[BX],
                                             const double (&a1)[BX], T* r0, T* r1)
{
    using P = typename Pair2<T>::type;
    static_assert(BX <= 32, "cases cover blocksizes up to 32");
    switch (count) {
        PSB_BOTTOM_CASE(2) PSB_BOTTOM_CASE(4) PSB_BOTTOM_CASE(6) PSB_BOTTOM_CASE(8)
        PSB_BOTTOM_CASE(10) PSB_BOTTOM_CASE(12) PSB_BOTTOM_CASE(14) PSB_BOTTOM_CASE(16)
        PSB_BOTTOM_CASE(18) PSB_BOTTOM_CASE(20) PSB_BOTTOM_CASE(22) PSB_BOTTOM_CASE(24)
        PSB_BOTTOM_CASE(26) PSB_BOTTOM_CASE(28) PSB_BOTTOM_CASE(30) PSB_BOTTOM_CASE(32)
        default: break;
    }
}
#undef PSB_BOTTOM_CASE

// Gap: rows K and K-1 of level m (K odd), in place and descending (row k
// reads old rows k-2, k-1, k).  On entry L1a, L1b hold the left neighbours
// of old rows K and K-1 (column 1 of the lane to the left, or the carry for
// lane 0); on exit those of old rows K-2 and K-3, which the next pair needs
// (old rows below K-1 are not written by this pair), so a pair takes four
// new shuffles.
template <int K, int BX, class T, int VAR = 0>
__device__ __forceinline__ void gap_pair(double (&a0)[BX], double (&a1)[BX], const double* cr0,
                                         int lane, double cr, double& L1a, double& L1b,
                                         const VarFields& vf = VarFields{}, double* vring = nullptr,
                                         int K0 = 0, int row0 = 0, int nx = 0, int ny = 0,
                                         int gm = 0, int gm1 = 0, bool valid = false)
{
    if constexpr (K >= 3 && K < BX) {
        const double L1d = L1a, L1c = L1b;
        const double2 cu = *reinterpret_cast<const double2*>(cr0 + (K - 2) * 2);
        const double L1u = from_left(a1[K - 2], cu.y, lane);
        const double L0c = from_left(a0[K - 1], cr0[(K - 1) * 2], lane);
        double n0, n1;
        if constexpr (VAR == 0) {
            heat_pair<T>(L1u, L1c, L1d, L0c, a0[K - 2], a0[K - 1], a0[K], a1[K - 1], cr, n0, n1);
        } else {
            // rows K, K-1 are ring positions K0-K, K0-K+1; the level's last
            // row is new index 2
            const VarPre p = var_next<VAR>(vf, vring, K0 - K, K - kVarAhead >= 2,
                                           gap_grid_row(row0, K - kVarAhead, nx), ny, gm, gm1, lane);
            heat_pair_var<VAR>(L1u, L1c, L1d, L0c, a0[K - 2], a0[K - 1], a0[K], a1[K - 1], p, vf,
                               gap_grid_row(row0, K, nx), ny, gm, gm1, valid, n0, n1);
        }
        a0[K] = n0;
        a1[K] = n1;
        // row K-1: up K-3, centre K-2, down K-1
        const double L1uu = from_left(a1[K - 3], cr0[(K - 3) * 2 + 1], lane);
        const double L0cc = from_left(a0[K - 2], cu.x, lane);
        if constexpr (VAR == 0) {
            heat_pair<T>(L1uu, L1u, L1c, L0cc, a0[K - 3], a0[K - 2], a0[K - 1], a1[K - 2], cr, n0,
                         n1);
        } else {
            const VarPre p = var_next<VAR>(vf, vring, K0 - K + 1, K - 1 - kVarAhead >= 2,
                                           gap_grid_row(row0, K - 1 - kVarAhead, nx), ny, gm, gm1,
                                           lane);
            heat_pair_var<VAR>(L1uu, L1u, L1c, L0cc, a0[K - 3], a0[K - 2], a0[K - 1], a1[K - 2],
                               p, vf, gap_grid_row(row0, K - 1, nx), ny, gm, gm1, valid, n0, n1);
        }
        a0[K - 1] = n0;
        a1[K - 1] = n1;
        L1a = L1u;
        L1b = L1uu;
    }
}

// Gap: the left neighbours of old rows K and K-1, which the level's first
// pair takes on entry.
template <int K, int BX, int VAR = 0>
__device__ __forceinline__ void gap_entry(const double (&a1)[BX], const double* cr0, int lane,
                                          double& L1a, double& L1b,
                                          const VarFields& vf = VarFields{},
                                          double* vring = nullptr, int row0 = 0, int nx = 0,
                                          int ny = 0, int gm = 0, int gm1 = 0)
{
    if constexpr (K >= 3 && K < BX) {
        if constexpr (VAR != 0) {  // ring positions 0 .. kVarAhead-1: rows K, K-1, ...
            constexpr int F = var_fields<VAR>() * 32;
#pragma unroll
            for (int q = 0; q < kVarAhead; ++q) {
                if (K - q >= 2) var_issue<VAR>(vf, vring + q * F, gap_grid_row(row0, K - q, nx), ny,
                                               gm, gm1, lane);
                cp_async_commit();
            }
        }
        L1a = from_left(a1[K], cr0[K * 2 + 1], lane);
        L1b = from_left(a1[K - 1], cr0[(K - 1) * 2 + 1], lane);
    }
}

// One column segment of one band, run by one warp; `unit` indexes the
// segment's y-faces; `carry` is the warp's own shared memory
// (heat_fast_warp_doubles: two packed carry buffers, then the ring).
// T: storage type of the fields and faces (double or float).
// MINROWS: rows every prism level is known to keep (BX - 2h for h levels per
// half-cycle); the row loop tests for the level's end only past them.
template <int BX, bool GAP, class T = double, int VAR = 0, int MINROWS = 2>
__device__ __forceinline__ void heat_fast_body(const SweptArgs& a, const SegGeom sg,
                                               const int unit, double* carry)
{
    static_assert(VAR == 0 || sizeof(T) == 8, "per-cell courant numbers on float64 fields");
    using P = typename Pair2<T>::type;
    constexpr int hx = BX / 2;
    const int lane = threadIdx.x & 31;
    const int H = a.H, Hm = a.Hmax, nx = a.nx, ny = a.ny;
    const int band = sg.band;
    const int r0 = GAP ? (a.off + band * BX - hx) : (a.off + band * BX);
    const int s0 = sg.s0;
    // segments are whole multiples of 32 columns: 64-column chunks, the last
    // one possibly 32 wide (lanes 16..31 then hold columns past the segment)
    const int wseg = sg.s1 - s0;
    const int nchunks = (wseg + kFastChunk - 1) / kFastChunk;
    const int lastw = wseg - (nchunks - 1) * kFastChunk;
    const double cr = a.p.d[0];
    // one packed carry buffer: level j's rows at carry_rows(j), 2 columns each
    const int CB = 2 * (carry_rows<BX, false>(Hm) > carry_rows<BX, true>(Hm)
                            ? carry_rows<BX, false>(Hm)
                            : carry_rows<BX, true>(Hm));
    T* ring = reinterpret_cast<T*>(carry + 2 * CB);  // gap: [kFaceSlots][4][32][2] of T
    // VAR: the per-cell operand ring, after the warp's base share
    double* vring = carry + heat_fast_warp_doubles<BX>(Hm);
    const int HF = Hm - 1;
    const int bup = wrap(band - 1, a.nb);
    const int r0w = wrap(r0, nx);

    double a0[BX], a1[BX];
    for (int c = 0; c < nchunks; ++c) {
        const int cw = s0 + c * kFastChunk;
        const bool first = (c == 0), last = (c == nchunks - 1);
        const int nact = last ? lastw / 2 : 32;  // lanes holding this chunk's columns
        double* cin = carry + (c & 1) * CB;
        double* cout = carry + ((c + 1) & 1) * CB;
        const int gcol = wrap(cw + 2 * lane, ny);  // the lane's level-0 column (x-face column)
        // ---- level 0 ------------------------------------------------------
        {
            const T* b = reinterpret_cast<const T*>(a.bin);  // its = 1: the only base level
            const int g = wrap(cw + 2 * lane, ny);
            auto rowp = [&](int r) {  // band row r, wrapped
                int row = r0w + r;
                row -= row >= nx ? nx : 0;
                return b + (size_t)row * ny;
            };
            if (!GAP) {
#pragma unroll
                for (int i = 0; i < BX; ++i) {
                    const double2 v = widen(*reinterpret_cast<const P*>(rowp(i) + g));
                    a0[i] = v.x;
                    a1[i] = v.y;
                }
            } else {
#pragma unroll
                for (int k = 0; k < 2; ++k) {
                    const double2 v = widen(*reinterpret_cast<const P*>(rowp(hx - 2 + k) + g));
                    a0[k] = v.x;
                    a1[k] = v.y;
                }
                const double2 v0 = widen(*reinterpret_cast<const P*>(rowp(hx) + g));
                const double2 v1 = widen(*reinterpret_cast<const P*>(rowp(hx + 1) + g));
                a0[2] = v0.x;
                a1[2] = v0.y;
                a0[3] = v1.x;
                a1[3] = v1.y;
            }
            // carry of level 0: columns cw-2 and cw-1 of the level's rows
            const int nrow0 = GAP ? 4 : BX;
            const int rbase = GAP ? hx - 2 : 0;
            const int gl = wrap(cw - 2, ny), gl1 = wrap(cw - 1, ny);
            for (int k = lane; k < nrow0; k += 32) {
                const T* src = rowp(rbase + k);
                cin[k * 2 + 0] = src[gl];
                cin[k * 2 + 1] = src[gl1];
            }
        }
        // gap: the face rows of levels 1 .. kFaceDepth start arriving; one
        // commit group per level, empty past the last level with faces
        if (GAP) {
#pragma unroll
            for (int d = 1; d <= kFaceDepth; ++d) {
                if (d <= H - 1) issue_faces(a, bup, band, HF, d, gcol, lane, ring + d * 256);
                cp_async_commit();
            }
        }
        __syncwarp();
        for (int m = 1; m <= H; ++m) {
            const double* cr0 = cin + carry_rows<BX, GAP>(m - 1) * 2;  // carry of level m-1
            const int gm = wrap(cw - m + 2 * lane, ny);  // this lane's first column at level m
            const int gm1 = gm + 1 == ny ? 0 : gm + 1;   // and its second
            const bool even = (m & 1) == 0;              // parity of gm (cw and ny are even)
            // left-seam mask: the first chunk's level m starts at column s0+m
            // (lane m); a 32-column last chunk ends at lane 15
            const bool valid = (!first || lane >= m) && lane < nact;
            // per-cell courant numbers: this level's slab of the Laplacians
            // (VAR 1 stores level gts-1, VAR 2 reads level LEN-gts) and the
            // adjoint's sum
            VarFields vf{};
            if constexpr (VAR != 0) {
                const long long gts = a.gts_base + a.L0 + m;
                vf.C = a.p.f[0];
                const long long lvl = VAR == 1 ? gts - 1 : a.p.i[3] - gts;
                vf.lu = a.p.f[1] ? a.p.f[1] + lvl * a.p.fs : nullptr;
                vf.g = a.p.f[2];
            }
            int nrow;  // rows of level m held in the arrays
            double2 lower2 = make_double2(0.0, 0.0), lower3 = lower2;  // gap: lower face rows
            if (!GAP) {
                // ---- prism: level m rows [m, BX-m) at indices [0, BX-2m) ----
                // old index i <-> row m-1+i; new index i <-> row m+i
                const int count = BX - 2 * m;
                nrow = count;
                const double2 cu = *reinterpret_cast<const double2*>(cr0 + 0);
                double2 cc = *reinterpret_cast<const double2*>(cr0 + 2);
                double L1u = from_left(a1[0], cu.y, lane);
                double L1c = from_left(a1[1], cc.y, lane);
                // VAR: grid row of band row m (new index 0); ring positions
                // 0 .. kVarAhead-1 start arriving
                int row = r0w + m;
                row -= row >= nx ? nx : 0;
                if constexpr (VAR != 0) {
                    constexpr int F = var_fields<VAR>() * 32;
#pragma unroll
                    for (int q = 0; q < kVarAhead; ++q) {
                        int rq = row + q;
                        rq -= rq >= nx ? nx : 0;
                        if (q < count) var_issue<VAR>(vf, vring + q * F, rq, ny, gm, gm1, lane);
                        cp_async_commit();
                    }
                }
#pragma unroll
                for (int i = 0; i < BX - 2; ++i) {
                    if (i >= MINROWS && i >= count) break;
                    const double2 cd = *reinterpret_cast<const double2*>(cr0 + (i + 2) * 2);
                    const double L1d = from_left(a1[i + 2], cd.y, lane);
                    const double L0c = from_left(a0[i + 1], cc.x, lane);
                    double n0, n1;
                    if constexpr (VAR == 0) {
                        heat_pair<T>(L1u, L1c, L1d, L0c, a0[i], a0[i + 1], a0[i + 2], a1[i + 1],
                                     cr, n0, n1);
                    } else {
                        int ra = row + kVarAhead;  // grid row of ring position i + kVarAhead
                        ra -= ra >= nx ? nx : 0;
                        const VarPre pc = var_next<VAR>(vf, vring, i, i + kVarAhead < count, ra, ny,
                                                        gm, gm1, lane);
                        heat_pair_var<VAR>(L1u, L1c, L1d, L0c, a0[i], a0[i + 1], a0[i + 2],
                                           a1[i + 1], pc, vf, row, ny, gm, gm1, valid, n0, n1);
                        row = row + 1 == nx ? 0 : row + 1;
                    }
                    a0[i] = n0;
                    a1[i] = n1;
                    L1u = L1c;
                    L1c = L1d;
                    cc = cd;
                }
            } else {
                // ---- level m rows [hx-m, hx+m) at indices [2, 2m+2) ----------
                // old index k <-> row hx-m-1+k for k < 2m+2 (indices 2m, 2m+1:
                // the lower prism's face rows, placed there at the end of the
                // previous level); new index k <-> row hx-m-2+k reads old rows
                // k-2 (up), k-1 (centre), k (down).
                const int K0 = 2 * m + 1;
                nrow = 2 * m + 2;
                // grid row of new index 0 (band row hx-m-2)
                int grow0 = r0w + hx - m - 2;
                grow0 += grow0 < 0 ? nx : 0;
                grow0 -= grow0 >= nx ? nx : 0;
                // rows K0 .. 2, entered at K0 = 2m+1 (a prologue places the
                // lower face rows of level m-1 and takes the first pair's two
                // carried neighbours) and falling through
                double L1a = 0.0, L1b = 0.0;
                const T* lower = ring + ((m - 1) % kFaceSlots) * 256 + 2 * 64 + lane * 2;
#define PSB_GAP_ENTRY(K)                                                                   \
    case K:                                                                                \
        gap_lower<K, BX, T>(a0, a1, lower);                                                \
        gap_entry<K, BX, VAR>(a1, cr0, lane, L1a, L1b, vf, vring, grow0, nx, ny, gm, gm1);   \
        goto pair_##K;
#define PSB_GAP_PAIR(K)                                                                    \
    pair_##K:                                                                              \
    gap_pair<K, BX, T, VAR>(a0, a1, cr0, lane, cr, L1a, L1b, vf, vring, K0, grow0, nx, ny,   \
                            gm, gm1, valid);
                switch (K0) {
                    PSB_GAP_ENTRY(31) PSB_GAP_ENTRY(29) PSB_GAP_ENTRY(27) PSB_GAP_ENTRY(25)
                    PSB_GAP_ENTRY(23) PSB_GAP_ENTRY(21) PSB_GAP_ENTRY(19) PSB_GAP_ENTRY(17)
                    PSB_GAP_ENTRY(15) PSB_GAP_ENTRY(13) PSB_GAP_ENTRY(11) PSB_GAP_ENTRY(9)
                    PSB_GAP_ENTRY(7) PSB_GAP_ENTRY(5) PSB_GAP_ENTRY(3)
                default:
                    goto pairs_done;
                }
                PSB_GAP_PAIR(31) PSB_GAP_PAIR(29) PSB_GAP_PAIR(27) PSB_GAP_PAIR(25)
                PSB_GAP_PAIR(23) PSB_GAP_PAIR(21) PSB_GAP_PAIR(19) PSB_GAP_PAIR(17)
                PSB_GAP_PAIR(15) PSB_GAP_PAIR(13) PSB_GAP_PAIR(11) PSB_GAP_PAIR(9)
                PSB_GAP_PAIR(7) PSB_GAP_PAIR(5) PSB_GAP_PAIR(3)
            pairs_done:
#undef PSB_GAP_ENTRY
#undef PSB_GAP_PAIR
                // the face rows of level m: the upper ones join at indices 0, 1;
                // the lower ones (indices 2m+2, 2m+3, the next level's first
                // centre and down rows) at the next level's entry, and in the
                // carry from here.  Each lane reads back only the pairs it
                // copied.
                if (m <= H - 1) {
                    cp_async_wait<kFaceDepth - 1>();  // level m's group has landed
                    const T* sl = ring + (m % kFaceSlots) * 256 + lane * 2;
                    const double2 f0 = widen(*reinterpret_cast<const P*>(sl + 0 * 64));
                    const double2 f1 = widen(*reinterpret_cast<const P*>(sl + 1 * 64));
                    lower2 = widen(*reinterpret_cast<const P*>(sl + 2 * 64));
                    lower3 = widen(*reinterpret_cast<const P*>(sl + 3 * 64));
                    a0[0] = f0.x;
                    a1[0] = f0.y;
                    a0[1] = f1.x;
                    a1[1] = f1.y;
                    // refill the slot of level m-1 (read one level ago)
                    const int mf = m + kFaceDepth;
                    if (mf <= H - 1)
                        issue_faces(a, bup, band, HF, mf, gcol, lane, ring + (mf % kFaceSlots) * 256);
                    cp_async_commit();
                }
            }
            if (m <= H - 1 && !last) {
                double* co = cout + carry_rows<BX, GAP>(m) * 2;
#pragma unroll
                for (int i = 0; i < BX; ++i) {
                    if (i >= nrow) break;
                    if (lane == 31)
                        *reinterpret_cast<double2*>(co + i * 2) = make_double2(a0[i], a1[i]);
                }
                // gap: the lower face rows complete the level's carry
                if (GAP && lane == 31) {
                    *reinterpret_cast<double2*>(co + nrow * 2) = lower2;
                    *reinterpret_cast<double2*>(co + nrow * 2 + 2) = lower3;
                }
            }
            // ---- outputs of level m ------------------------------------------
            // computed rows: prism indices [0, nrow) (band rows m+i); gap
            // indices [2, nrow) (band rows hx-m-2+k)
            const int ibeg = GAP ? 2 : 0;
            const int rfirst = GAP ? hx - m - 2 : m;  // band row of index 0
            if (!GAP && m <= H - 1 && valid) {
                // faces are stored at the chunk's level-0 columns (xface_col)
                const size_t fb = ((size_t)band * HF + (m - 1)) * 2;
                T* xf = reinterpret_cast<T*>(a.xface) + gcol;
                *reinterpret_cast<P*>(xf + ((fb + 0) * 2 + 0) * ny) = pair2<T>(a0[0], a1[0]);
                *reinterpret_cast<P*>(xf + ((fb + 0) * 2 + 1) * ny) = pair2<T>(a0[1], a1[1]);
                store_bottom<BX, T>(BX - 2 * m, a0, a1, xf + ((fb + 1) * 2 + 0) * ny,
                                    xf + ((fb + 1) * 2 + 1) * ny);
            }
            const long long fs = frame_slot(a, a.L0 + m);
            if (m == H || fs >= 0) {
                T* fr = fs >= 0 ? reinterpret_cast<T*>(a.frames) + (size_t)fs * nx * ny : nullptr;
                T* bo = reinterpret_cast<T*>(a.bout);
#pragma unroll
                for (int i = 0; i < BX; ++i) {
                    if (i >= nrow) break;
                    if (i < ibeg) continue;
                    int row = r0w + rfirst + i;
                    row -= row >= nx ? nx : 0;
                    const size_t o = (size_t)row * ny;
                    if (m == H && valid) st_pair<T>(bo + o, gm, gm1, a0[i], a1[i], even);
                    if (fr && valid) st_pair<T>(fr + o, gm, gm1, a0[i], a1[i], even);
                }
            }
            // VAR 2: the next level updates this level's sums from other lanes
            if constexpr (VAR == 2) __syncwarp();
            // y-faces at the segment's column edges (read by the seam kernels)
            if (m <= H - 1 && (first || last)) {
#pragma unroll
                for (int side = 0; side < 2; ++side) {
                    if ((side == 0 && !first) || (side == 1 && !last)) continue;
                    const int owner = side == 0 ? m : nact - 1;
                    T* yf = reinterpret_cast<T*>(a.yface) +
                            (((size_t)unit * 2 + side) * HF + (m - 1)) * BX * 2;
#pragma unroll
                    for (int i = 0; i < BX; ++i) {
                        if (i >= nrow) break;
                        if (i < ibeg) continue;
                        if (lane == owner)
                            *reinterpret_cast<P*>(yf + (rfirst + i) * 2) = pair2<T>(a0[i], a1[i]);
                    }
                }
            }
        }
        __syncwarp();
    }
}

// VAR 0: heat (one courant number); VAR 1: a courant number per cell
// (HeatVar), storing each old level's Laplacian when p.f[1] is set; VAR 2: the
// adjoint in mu = C .* lambda (HeatVarAdjMu).
template <int BX, bool GAP, class T = double, int VAR = 0, int MINROWS = 2>
__global__ void __launch_bounds__(32 * kFastWarps, kFastCtasPerSm<BX, VAR>) heat_stream_fast(SweptArgs a)
{
    extern __shared__ double sm[];
    const int warp = threadIdx.x >> 5;
    const int unit = blockIdx.x * kFastWarps + warp;
    if (unit >= a.nb * a.nseg) return;  // whole warp leaves together
    heat_fast_body<BX, GAP, T, VAR, MINROWS>(a, seg_geom(a, unit), unit,
                                    sm + (size_t)warp * heat_fast_warp_doubles_v<BX, VAR>(a.Hmax));
}

}  // namespace psb
