// Heat equation with a spatially varying diffusivity and its adjoint.
//
// Forward, per cell (the heat plugin's operation order, pysweep/equations/
// heat.py:60-64, with the courant number per cell):
//     C = alpha * dt / dx / dx
//     u' = (C*((u[x+1]-2u)+u[x-1]) + C*((u[y+1]-2u)+u[y-1])) + u
// i.e. u_{n+1} = u_n + C .* (L u_n) with L the periodic 5-point Laplacian
// (symmetric).  For J(u_N), with lambda_n = dJ/du_n:
//     lambda_n = lambda_{n+1} + L (C .* lambda_{n+1})
//     dJ/dC   += lambda_{n+1} .* (L u_n),        dJ/dalpha = dJ/dC * dt/dx/dx
// The forward stores u every `every` steps; the backward pass walks the
// segments from the last to the first, recomputes the segment's states from
// its checkpoint into a work buffer, then runs the adjoint steps backward
// through the segment.
//
// All kernels stream 64-column strips down blocks of rows: lane l holds
// columns 2l, 2l+1, the rows above/at/below in registers, lateral neighbours
// by shuffle (the layout of heat_standard_fast).  The backward pass fuses two
// time steps per launch, both in the recompute (u_n -> u_{n+1}, u_{n+2}) and
// in the adjoint (lambda_{n+1} -> lambda_{n-1}, gradient of both steps added
// with one read and one write of dJ/dC): the first step is also evaluated on
// one halo row above and below the strip and one halo column either side, so
// the second step finds its neighbours in registers.  Every cell sees the
// same operations in the same order as in the one-step kernels, so fused and
// unfused passes agree bitwise.  Operand rows reach each warp through a
// cp.async ring in shared memory three rows ahead of use (RowRing), which
// keeps enough loads in flight at the occupancy the register use allows.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>

#include "../../include/pysweep_b200.h"
#include "heat_fast.cuh"

namespace psb {
namespace {

struct Strip {
    int nx, ny, g, x0, xend, lane, hcol, hcol2;
    __device__ Strip(int nx_, int ny_, int rows) : nx(nx_), ny(ny_)
    {
        const int warp = threadIdx.x >> 5;
        lane = threadIdx.x & 31;
        const int cw = (blockIdx.x * 8 + warp) * 64;
        g = cw + 2 * lane;
        x0 = blockIdx.y * rows;
        xend = min(x0 + rows, nx);
        // halo columns: lane 0 holds cw-1 and cw-2, lane 31 cw+64 and cw+65 (periodic)
        const int gl = cw == 0 ? ny - 1 : cw - 1;
        const int gl2 = gl == 0 ? ny - 1 : gl - 1;
        const int gr = cw + 64 == ny ? 0 : cw + 64;
        const int gr2 = gr + 1 == ny ? 0 : gr + 1;
        hcol = lane == 0 ? gl : gr;
        hcol2 = lane == 0 ? gl2 : gr2;
    }
    __device__ bool active() const { return g - 2 * lane < ny; }
    __device__ bool edge() const { return lane == 0 || lane == 31; }
    __device__ size_t row(int x) const
    {
        x += x < 0 ? nx : 0;
        x -= x >= nx ? nx : 0;
        return (size_t)x * ny;
    }
};

// values of one row at this lane's pair plus the halo column for lanes 0/31
struct Row {
    double a, b, h;
};

// a row with the second halo column too (h2: cw-2 on lane 0, cw+65 on lane 31)
struct Row2 {
    double a, b, h, h2;
    __device__ Row row() const { return Row{a, b, h}; }
};

__device__ __forceinline__ Row load_row(const double* f, const Strip& s, int x)
{
    const double* p = f + s.row(x);
    const double2 v = *reinterpret_cast<const double2*>(p + s.g);
    Row r;
    r.a = v.x;
    r.b = v.y;
    r.h = s.edge() ? p[s.hcol] : 0.0;
    return r;
}

__device__ __forceinline__ Row2 load_row2(const double* f, const Strip& s, int x)
{
    const double* p = f + s.row(x);
    const double2 v = *reinterpret_cast<const double2*>(p + s.g);
    Row2 r;
    r.a = v.x;
    r.b = v.y;
    r.h = s.edge() ? p[s.hcol] : 0.0;
    r.h2 = s.edge() ? p[s.hcol2] : 0.0;
    return r;
}

__device__ __forceinline__ Row2 mul_row2(const Row2& c, const Row2& l)
{
    return Row2{__dmul_rn(c.a, l.a), __dmul_rn(c.b, l.b), __dmul_rn(c.h, l.h),
                __dmul_rn(c.h2, l.h2)};
}

__device__ __forceinline__ void store_pair(double* f, const Strip& s, int x, double v0, double v1)
{
    *reinterpret_cast<double2*>(f + s.row(x) + s.g) = make_double2(v0, v1);
}

// 5-point operator ((f[x+1]-2f)+f[x-1]) + ((f[y+1]-2f)+f[y-1]) for the pair
__device__ __forceinline__ void lap(const Row& up, const Row& c, const Row& dn, int lane,
                                    double& l0, double& l1)
{
    double left = __shfl_up_sync(0xffffffffu, c.b, 1);
    double right = __shfl_down_sync(0xffffffffu, c.a, 1);
    if (lane == 0) left = c.h;
    if (lane == 31) right = c.h;
    l0 = __dadd_rn(__dadd_rn(__fma_rn(-2.0, c.a, dn.a), up.a),
                   __dadd_rn(__fma_rn(-2.0, c.a, c.b), left));
    l1 = __dadd_rn(__dadd_rn(__fma_rn(-2.0, c.b, dn.b), up.b),
                   __dadd_rn(__fma_rn(-2.0, c.b, right), c.a));
}

// the same operator on the halo column of lanes 0 (cw-1) and 31 (cw+64)
__device__ __forceinline__ double lap_halo(const Row2& up, const Row2& c, const Row2& dn, int lane)
{
    const double left = lane == 0 ? c.h2 : c.b;
    const double right = lane == 0 ? c.a : c.h2;
    return __dadd_rn(__dadd_rn(__fma_rn(-2.0, c.h, dn.h), up.h),
                     __dadd_rn(__fma_rn(-2.0, c.h, right), left));
}

// one forward step at the pair
__device__ __forceinline__ void fe_pair(const Row& up, const Row& c, const Row& dn, double ca,
                                        double cb, int lane, double& n0, double& n1)
{
    double left = __shfl_up_sync(0xffffffffu, c.b, 1);
    double right = __shfl_down_sync(0xffffffffu, c.a, 1);
    if (lane == 0) left = c.h;
    if (lane == 31) right = c.h;
    n0 = heat_fe(c.a, up.a, dn.a, left, c.b, ca);
    n1 = heat_fe(c.b, up.b, dn.b, c.a, right, cb);
}

// one forward step on the halo column
__device__ __forceinline__ double fe_halo(const Row2& up, const Row2& c, const Row2& dn, double ch,
                                          int lane)
{
    const double ym = lane == 0 ? c.h2 : c.b;
    const double yp = lane == 0 ? c.a : c.h2;
    return heat_fe(c.h, up.h, dn.h, ym, yp, ch);
}

__global__ void courant_kernel(const double* __restrict__ alpha, double* __restrict__ C, size_t n,
                               double dt, double dx)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        C[i] = alpha[i] * dt / dx / dx;
}

// ---- operand rings ---------------------------------------------------------
// Every kernel below streams a strip down its rows; iteration t needs a few
// rows of its operands.  A warp copies them with cp.async into a ring of
// kRingSlots slots kRingDepth iterations before they are used, so loads stay
// in flight without holding registers.  A slot holds P 16-byte pairs per lane
// ([P][32 lanes][2]) and HH halo values for the edge lanes 0 and 31
// ([HH][2]).  Each lane reads back only what it copied; a slot is refilled
// one iteration after it was read.
constexpr int kRingDepth = 3;
constexpr int kRingSlots = kRingDepth + 1;

template <int P, int HH>
struct RowRing {
    static constexpr int kSlot = P * 64 + HH * 2;  // doubles per slot
    static constexpr size_t smem(int warps) { return sizeof(double) * warps * kRingSlots * kSlot; }
    double* base;
    int lane, edge;  // edge: 0 for lane 0, 1 for lane 31
    __device__ RowRing(double* sm, const Strip& s)
        : base(sm + (threadIdx.x >> 5) * kRingSlots * kSlot), lane(s.lane), edge(s.lane == 31)
    {
    }
    __device__ double* slot(int t) const { return base + (t % kRingSlots) * kSlot; }
    __device__ void pair(double* sl, int f, const double* src) const
    {
        cp_async16(sl + (f * 32 + lane) * 2, src);
    }
    __device__ void halo(double* sl, int h, const double* src) const
    {
        cp_async8(sl + P * 64 + h * 2 + edge, src);
    }
    __device__ double2 get_pair(const double* sl, int f) const
    {
        return *reinterpret_cast<const double2*>(sl + (f * 32 + lane) * 2);
    }
    __device__ double get_halo(const double* sl, int h, bool on) const
    {
        return on ? sl[P * 64 + h * 2 + edge] : 0.0;
    }
};

// u' = (C*dxx + C*dyy) + u.  Iteration x (rows x0 .. xend-1): u row x+1, C row x.
// LAP: also store the old level's Laplacian (dxx + dyy before the courant
// factor, the order of lap()) at lap_out.
template <bool LAP = false>
__global__ void __launch_bounds__(256) heatvar_step(const double* __restrict__ u,
                                                    const double* __restrict__ C,
                                                    double* __restrict__ out, int nx, int ny,
                                                    int rows, double* __restrict__ lap_out = nullptr)
{
    extern __shared__ double ring_sm[];
    const Strip s(nx, ny, rows);
    if (!s.active()) return;
    using Ring = RowRing<2, 1>;
    const Ring R(ring_sm, s);
    const int n = s.xend - s.x0;
    auto issue = [&](int t) {
        if (t < n) {
            double* sl = R.slot(t);
            const size_t r1 = s.row(s.x0 + t + 1);
            R.pair(sl, 0, u + r1 + s.g);
            R.pair(sl, 1, C + s.row(s.x0 + t) + s.g);
            if (s.edge()) R.halo(sl, 0, u + r1 + s.hcol);
        }
        cp_async_commit();
    };
    for (int t = 0; t < kRingDepth; ++t) issue(t);
    Row up = load_row(u, s, s.x0 - 1), ce = load_row(u, s, s.x0);
    for (int t = 0; t < n; ++t) {
        cp_async_wait<kRingDepth - 1>();
        const double* sl = R.slot(t);
        const double2 dv = R.get_pair(sl, 0), cr = R.get_pair(sl, 1);
        const Row dn{dv.x, dv.y, R.get_halo(sl, 0, s.edge())};
        issue(t + kRingDepth);
        double n0, n1;
        fe_pair(up, ce, dn, cr.x, cr.y, s.lane, n0, n1);
        store_pair(out, s, s.x0 + t, n0, n1);
        if (LAP) {
            double l0, l1;
            lap(up, ce, dn, s.lane, l0, l1);
            store_pair(lap_out, s, s.x0 + t, l0, l1);
        }
        up = ce;
        ce = dn;
    }
}

// Two forward steps: mid = step(u), out = step(mid).  The first step runs on
// rows x0-1 .. xend and on the halo columns.  Iteration i = x0-1+t: u row i+1
// (two halo columns), C row i+1.
// LAP: instead of the middle state, store the Laplacians of the two old
// levels (u at lap_a, the middle state at lap_b).
template <bool LAP = false>
__global__ void __launch_bounds__(256) heatvar_step2(const double* __restrict__ u,
                                                     const double* __restrict__ C,
                                                     double* __restrict__ mid,
                                                     double* __restrict__ out, int nx, int ny,
                                                     int rows, double* __restrict__ lap_a = nullptr,
                                                     double* __restrict__ lap_b = nullptr)
{
    extern __shared__ double ring_sm[];
    const Strip s(nx, ny, rows);
    if (!s.active()) return;
    using Ring = RowRing<2, 3>;
    const Ring R(ring_sm, s);
    const int n = s.xend - s.x0 + 2;  // iterations i = x0-1 .. xend
    auto issue = [&](int t) {
        if (t < n) {
            double* sl = R.slot(t);
            const size_t r1 = s.row(s.x0 + t);  // row i+1
            R.pair(sl, 0, u + r1 + s.g);
            R.pair(sl, 1, C + r1 + s.g);
            if (s.edge()) {
                R.halo(sl, 0, u + r1 + s.hcol);
                R.halo(sl, 1, u + r1 + s.hcol2);
                R.halo(sl, 2, C + r1 + s.hcol);
            }
        }
        cp_async_commit();
    };
    for (int t = 0; t < kRingDepth; ++t) issue(t);
    Row2 uu = load_row2(u, s, s.x0 - 2), uc = load_row2(u, s, s.x0 - 1);
    Row cc = load_row(C, s, s.x0 - 1);
    Row cp{0.0, 0.0, 0.0};  // C one row up (own columns)
    Row mu{0.0, 0.0, 0.0}, mc{0.0, 0.0, 0.0};  // first-step rows i-2, i-1
    for (int t = 0; t < n; ++t) {
        const int i = s.x0 - 1 + t;
        cp_async_wait<kRingDepth - 1>();
        const double* sl = R.slot(t);
        const double2 uv = R.get_pair(sl, 0), cv = R.get_pair(sl, 1);
        const Row2 ud{uv.x, uv.y, R.get_halo(sl, 0, s.edge()), R.get_halo(sl, 1, s.edge())};
        const Row cn{cv.x, cv.y, R.get_halo(sl, 2, s.edge())};
        issue(t + kRingDepth);
        Row m;
        fe_pair(uu.row(), uc.row(), ud.row(), cc.a, cc.b, s.lane, m.a, m.b);
        m.h = fe_halo(uu, uc, ud, cc.h, s.lane);
        if (i >= s.x0 && i < s.xend) {
            if (LAP) {
                double l0, l1;
                lap(uu.row(), uc.row(), ud.row(), s.lane, l0, l1);
                store_pair(lap_a, s, i, l0, l1);
            } else {
                store_pair(mid, s, i, m.a, m.b);
            }
        }
        if (i > s.x0) {
            double o0, o1;
            fe_pair(mu, mc, m, cp.a, cp.b, s.lane, o0, o1);
            store_pair(out, s, i - 1, o0, o1);
            if (LAP) {
                double l0, l1;
                lap(mu, mc, m, s.lane, l0, l1);
                store_pair(lap_b, s, i - 1, l0, l1);
            }
        }
        uu = uc;
        uc = ud;
        cp = cc;
        cc = cn;
        mu = mc;
        mc = m;
    }
}

// One adjoint level: lam_out = lam + L(C .* lam);  gC += lam .* L(u).
// Iteration x: lam, C and u rows x+1 (halo column), lam and gC rows x.
__global__ void __launch_bounds__(256) heatvar_adjoint(const double* __restrict__ lam,
                                                       const double* __restrict__ C,
                                                       const double* __restrict__ u,
                                                       double* __restrict__ lam_out,
                                                       double* __restrict__ gC, int nx, int ny,
                                                       int rows)
{
    extern __shared__ double ring_sm[];
    const Strip s(nx, ny, rows);
    if (!s.active()) return;
    using Ring = RowRing<5, 3>;
    const Ring R(ring_sm, s);
    const int n = s.xend - s.x0;
    auto issue = [&](int t) {
        if (t < n) {
            double* sl = R.slot(t);
            const size_t r1 = s.row(s.x0 + t + 1), r0 = s.row(s.x0 + t);
            R.pair(sl, 0, lam + r1 + s.g);
            R.pair(sl, 1, C + r1 + s.g);
            R.pair(sl, 2, u + r1 + s.g);
            R.pair(sl, 3, lam + r0 + s.g);
            R.pair(sl, 4, gC + r0 + s.g);
            if (s.edge()) {
                R.halo(sl, 0, lam + r1 + s.hcol);
                R.halo(sl, 1, C + r1 + s.hcol);
                R.halo(sl, 2, u + r1 + s.hcol);
            }
        }
        cp_async_commit();
    };
    for (int t = 0; t < kRingDepth; ++t) issue(t);
    auto mu_of = [](const Row& c, const Row& l) {
        return Row{__dmul_rn(c.a, l.a), __dmul_rn(c.b, l.b), __dmul_rn(c.h, l.h)};
    };
    Row mup = mu_of(load_row(C, s, s.x0 - 1), load_row(lam, s, s.x0 - 1));
    Row mce = mu_of(load_row(C, s, s.x0), load_row(lam, s, s.x0));
    Row uup = load_row(u, s, s.x0 - 1), uce = load_row(u, s, s.x0);
    for (int t = 0; t < n; ++t) {
        const int x = s.x0 + t;
        cp_async_wait<kRingDepth - 1>();
        const double* sl = R.slot(t);
        const double2 lv = R.get_pair(sl, 0), cv = R.get_pair(sl, 1), uv = R.get_pair(sl, 2);
        const double2 l = R.get_pair(sl, 3), gc = R.get_pair(sl, 4);
        const Row ldn{lv.x, lv.y, R.get_halo(sl, 0, s.edge())};
        const Row cdn{cv.x, cv.y, R.get_halo(sl, 1, s.edge())};
        const Row udn{uv.x, uv.y, R.get_halo(sl, 2, s.edge())};
        issue(t + kRingDepth);
        const Row mdn = mu_of(cdn, ldn);
        double lm0, lm1, lu0, lu1;
        lap(mup, mce, mdn, s.lane, lm0, lm1);
        lap(uup, uce, udn, s.lane, lu0, lu1);
        store_pair(lam_out, s, x, __dadd_rn(l.x, lm0), __dadd_rn(l.y, lm1));
        store_pair(gC, s, x, __fma_rn(l.x, lu0, gc.x), __fma_rn(l.y, lu1, gc.y));
        mup = mce;
        mce = mdn;
        uup = uce;
        uce = udn;
    }
}

// Two adjoint levels: from lam = lambda_{n+1}, u_hi = u_n and u_lo = u_{n-1},
//     lambda_n     = lam + L(C .* lam)            (rows x0-1 .. xend, halo columns)
//     lambda_{n-1} = lambda_n + L(C .* lambda_n)  -> lam_out
//     gC += lam .* L(u_hi);  gC += lambda_n .* L(u_lo)   (one read, one write)
// Iteration i = x0-1+t evaluates the first level at row i and the second at
// row i-1; it needs lam, C, u_hi rows i+1 and u_lo, gC rows i.  (gC row i is
// written one iteration after it is read, by this warp only.)
__global__ void __launch_bounds__(256) heatvar_adjoint2(
    const double* __restrict__ lam, const double* __restrict__ C, const double* __restrict__ u_hi,
    const double* __restrict__ u_lo, double* __restrict__ lam_out, double* __restrict__ gC, int nx,
    int ny, int rows)
{
    extern __shared__ double ring_sm[];
    const Strip s(nx, ny, rows);
    if (!s.active()) return;
    using Ring = RowRing<5, 6>;
    const Ring R(ring_sm, s);
    const int n = s.xend - s.x0 + 2;  // iterations i = x0-1 .. xend
    auto issue = [&](int t) {
        if (t < n) {
            double* sl = R.slot(t);
            const size_t r1 = s.row(s.x0 + t), r0 = s.row(s.x0 - 1 + t);  // rows i+1, i
            R.pair(sl, 0, lam + r1 + s.g);
            R.pair(sl, 1, C + r1 + s.g);
            R.pair(sl, 2, u_hi + r1 + s.g);
            R.pair(sl, 3, u_lo + r0 + s.g);
            R.pair(sl, 4, gC + r0 + s.g);
            if (s.edge()) {
                R.halo(sl, 0, lam + r1 + s.hcol);
                R.halo(sl, 1, lam + r1 + s.hcol2);
                R.halo(sl, 2, C + r1 + s.hcol);
                R.halo(sl, 3, C + r1 + s.hcol2);
                R.halo(sl, 4, u_hi + r1 + s.hcol);
                R.halo(sl, 5, u_lo + r0 + s.hcol);
            }
        }
        cp_async_commit();
    };
    for (int t = 0; t < kRingDepth; ++t) issue(t);
    Row2 lc = load_row2(lam, s, s.x0 - 1), cc = load_row2(C, s, s.x0 - 1);
    Row2 m1u = mul_row2(load_row2(C, s, s.x0 - 2), load_row2(lam, s, s.x0 - 2));
    Row2 m1c = mul_row2(cc, lc);
    Row hu = load_row(u_hi, s, s.x0 - 1), hc = load_row(u_hi, s, s.x0);
    Row lu = load_row(u_lo, s, s.x0 - 1), lcur = load_row(u_lo, s, s.x0);
    Row m0u{0.0, 0.0, 0.0}, m0c{0.0, 0.0, 0.0};  // C .* lambda_n, rows i-2, i-1
    double ln0 = 0.0, ln1 = 0.0;                  // lambda_n at row i-1
    double g0 = 0.0, g1 = 0.0;                    // gC after the first level, row i-1
    for (int t = 0; t < n; ++t) {
        const int i = s.x0 - 1 + t;
        cp_async_wait<kRingDepth - 1>();
        const double* sl = R.slot(t);
        const bool e = s.edge();
        const double2 lv = R.get_pair(sl, 0), cv = R.get_pair(sl, 1), hv = R.get_pair(sl, 2);
        const double2 wv = R.get_pair(sl, 3), gold = R.get_pair(sl, 4);
        const Row2 ld{lv.x, lv.y, R.get_halo(sl, 0, e), R.get_halo(sl, 1, e)};
        const Row2 cd{cv.x, cv.y, R.get_halo(sl, 2, e), R.get_halo(sl, 3, e)};
        const Row hd{hv.x, hv.y, R.get_halo(sl, 4, e)};
        const Row ldn{wv.x, wv.y, R.get_halo(sl, 5, e)};
        issue(t + kRingDepth);
        const Row2 m1d = mul_row2(cd, ld);
        // first level at row i
        double a0, a1;
        lap(m1u.row(), m1c.row(), m1d.row(), s.lane, a0, a1);
        const double ah = lap_halo(m1u, m1c, m1d, s.lane);
        const Row ln{__dadd_rn(lc.a, a0), __dadd_rn(lc.b, a1), __dadd_rn(lc.h, ah)};
        const Row m0{__dmul_rn(cc.a, ln.a), __dmul_rn(cc.b, ln.b), __dmul_rn(cc.h, ln.h)};
        double ng0 = 0.0, ng1 = 0.0;
        if (i >= s.x0 && i < s.xend) {
            double q0, q1;
            lap(hu, hc, hd, s.lane, q0, q1);
            ng0 = __fma_rn(lc.a, q0, gold.x);
            ng1 = __fma_rn(lc.b, q1, gold.y);
            hu = hc;
            hc = hd;
        }
        // second level at row i-1
        if (i > s.x0) {
            double b0, b1, q0, q1;
            lap(m0u, m0c, m0, s.lane, b0, b1);
            lap(lu, lcur, ldn, s.lane, q0, q1);
            store_pair(lam_out, s, i - 1, __dadd_rn(ln0, b0), __dadd_rn(ln1, b1));
            store_pair(gC, s, i - 1, __fma_rn(ln0, q0, g0), __fma_rn(ln1, q1, g1));
            lu = lcur;
            lcur = ldn;
        }
        m1u = m1c;
        m1c = m1d;
        lc = ld;
        cc = cd;
        m0u = m0c;
        m0c = m0;
        ln0 = ln.a;
        ln1 = ln.b;
        g0 = ng0;
        g1 = ng1;
    }
}

__global__ void scale_kernel(double* __restrict__ g, size_t n, double f)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        g[i] *= f;
}

// Rows per strip: 64, halved (down to 8) while the grid has fewer warps than
// `per_sm` per SM of a 148-SM part.  Each kernel streams its strip row after
// row, so a kernel that fits many warps per SM (few registers) wants many
// short strips, one with few warps per SM wants tall strips (less halo work).
int adj_rows(int nx, int ny, int per_sm)
{
    int rows = 64;
    while (rows > 8 && (long long)(ny / 64) * ((nx + rows - 1) / rows) < 148LL * per_sm) rows /= 2;
    return rows;
}

dim3 strip_grid(int nx, int ny, int rows)
{
    return dim3((ny / 64 + 7) / 8, (nx + rows - 1) / rows);
}

// shared memory of the ring-fed kernels (8 warps per CTA)
constexpr size_t kStepSmem = RowRing<2, 1>::smem(8);
constexpr size_t kStep2Smem = RowRing<2, 3>::smem(8);
constexpr size_t kAdjSmem = RowRing<5, 3>::smem(8);
constexpr size_t kAdj2Smem = RowRing<5, 6>::smem(8);

cudaError_t allow_ring_smem()
{
    cudaError_t e = cudaFuncSetAttribute(heatvar_adjoint, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kAdjSmem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(heatvar_adjoint2, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kAdj2Smem);
    return e;
}

}  // namespace
}  // namespace psb

using namespace psb;

namespace {
int adj_check(int nx, int ny, char* err, size_t errlen)
{
    if (nx < 3 || ny < 64 || ny % 64) {
        if (err && errlen) snprintf(err, errlen, "need nx >= 3 and ny a multiple of 64 (got %dx%d)", nx, ny);
        return PS_ERR_INVALID;
    }
    return PS_OK;
}

int adj_cuda(cudaError_t e, char* err, size_t errlen)
{
    if (e == cudaSuccess) return PS_OK;
    if (err && errlen) snprintf(err, errlen, "%s", cudaGetErrorString(e));
    return PS_ERR_CUDA;
}
}  // namespace

extern "C" int ps_heatvar_courant(const double* d_alpha, double* d_courant, int nx, int ny,
                                  double dt, double dx, void* stream, char* err, size_t errlen)
{
    int rc = adj_check(nx, ny, err, errlen);
    if (rc) return rc;
    if (!d_alpha || !d_courant) {
        if (err && errlen) snprintf(err, errlen, "bad arguments");
        return PS_ERR_INVALID;
    }
    courant_kernel<<<1024, 256, 0, (cudaStream_t)stream>>>(d_alpha, d_courant, (size_t)nx * ny, dt,
                                                          dx);
    return adj_cuda(cudaGetLastError(), err, errlen);
}

extern "C" int ps_heatvar_recompute(const double* d_courant, const double* d_u0, double* d_lap,
                                    int length, int nx, int ny, double* d_work, void* stream,
                                    char* err, size_t errlen)
{
    int rc = adj_check(nx, ny, err, errlen);
    if (rc) return rc;
    if (!d_courant || !d_u0 || !d_lap || !d_work || length < 0) {
        if (err && errlen) snprintf(err, errlen, "bad arguments");
        return PS_ERR_INVALID;
    }
    cudaStream_t st = (cudaStream_t)stream;
    const size_t n = (size_t)nx * ny;
    const int rows = adj_rows(nx, ny, 8), rows_1 = adj_rows(nx, ny, 16);
    const dim3 grid = strip_grid(nx, ny, rows), grid_1 = strip_grid(nx, ny, rows_1);
    // two levels per launch (their Laplacians, then the state two levels on),
    // the states ping-pong through the two work fields
    const double* in = d_u0;
    int w = 0, j = 0;
    for (; j + 1 < length; j += 2) {
        double* out = d_work + (size_t)w * n;
        heatvar_step2<true><<<grid, 256, kStep2Smem, st>>>(in, d_courant, nullptr, out, nx, ny, rows,
                                                          d_lap + (size_t)j * n,
                                                          d_lap + (size_t)(j + 1) * n);
        in = out;
        w ^= 1;
    }
    if (j < length)
        heatvar_step<true><<<grid_1, 256, kStepSmem, st>>>(in, d_courant, d_work + (size_t)w * n, nx,
                                                          ny, rows_1, d_lap + (size_t)j * n);
    return adj_cuda(cudaGetLastError(), err, errlen);
}

extern "C" int ps_heatvar_forward(const double* d_u0, const double* d_alpha, double* d_uT, int nx,
                                  int ny, int64_t nsteps, double dt, double dx, double* d_courant,
                                  double* d_work, double* d_checkpoints, int every, void* stream,
                                  char* err, size_t errlen)
{
    int rc = adj_check(nx, ny, err, errlen);
    if (rc) return rc;
    if (!d_u0 || !d_alpha || !d_uT || !d_courant || !d_work || nsteps < 0 || every < 1) {
        if (err && errlen) snprintf(err, errlen, "bad arguments");
        return PS_ERR_INVALID;
    }
    cudaStream_t st = (cudaStream_t)stream;
    const size_t n = (size_t)nx * ny;
    const int rows = adj_rows(nx, ny, 48);  // heatvar_step: 40 registers
    courant_kernel<<<1024, 256, 0, st>>>(d_alpha, d_courant, n, dt, dx);
    // ping-pong between d_work and d_uT so that the last step lands in d_uT
    const double* in = d_u0;
    if (d_checkpoints)
        if ((rc = adj_cuda(cudaMemcpyAsync(d_checkpoints, d_u0, n * sizeof(double),
                                           cudaMemcpyDeviceToDevice, st), err, errlen)))
            return rc;
    if (nsteps == 0)
        return adj_cuda(cudaMemcpyAsync(d_uT, d_u0, n * sizeof(double), cudaMemcpyDeviceToDevice, st),
                        err, errlen);
    for (int64_t k = 0; k < nsteps; ++k) {
        double* out = ((nsteps - 1 - k) % 2 == 0) ? d_uT : d_work;
        heatvar_step<false><<<strip_grid(nx, ny, rows), 256, kStepSmem, st>>>(in, d_courant, out, nx, ny,
                                                                       rows);
        if (d_checkpoints && (k + 1) % every == 0 && k + 1 < nsteps)
            if ((rc = adj_cuda(cudaMemcpyAsync(d_checkpoints + (size_t)((k + 1) / every) * n, out,
                                               n * sizeof(double), cudaMemcpyDeviceToDevice, st),
                               err, errlen)))
                return rc;
        in = out;
    }
    return adj_cuda(cudaGetLastError(), err, errlen);
}

extern "C" int ps_heatvar_adjoint(const double* d_courant, const double* d_checkpoints, int every,
                                  const double* d_lamT, double* d_lam0, double* d_galpha, int nx,
                                  int ny, int64_t nsteps, double dt, double dx, double* d_states,
                                  double* d_lamwork, void* stream, char* err, size_t errlen)
{
    int rc = adj_check(nx, ny, err, errlen);
    if (rc) return rc;
    if (!d_courant || !d_checkpoints || !d_lamT || !d_lam0 || !d_galpha || !d_states ||
        !d_lamwork || every < 1 || nsteps < 0) {
        if (err && errlen) snprintf(err, errlen, "bad arguments");
        return PS_ERR_INVALID;
    }
    cudaStream_t st = (cudaStream_t)stream;
    const size_t n = (size_t)nx * ny;
    const int rows = adj_rows(nx, ny, 8);      // heatvar_step2: 80 registers
    const int rows_a = adj_rows(nx, ny, 8);    // heatvar_adjoint2: 128 registers
    const int rows_1 = adj_rows(nx, ny, 16);   // heatvar_step, heatvar_adjoint
    const dim3 grid = strip_grid(nx, ny, rows), grid_a = strip_grid(nx, ny, rows_a);
    const dim3 grid_1 = strip_grid(nx, ny, rows_1);
    const int64_t nseg = (nsteps + every - 1) / every;
    if ((rc = adj_cuda(allow_ring_smem(), err, errlen))) return rc;
    // adjoint launches: two levels per launch, one more for an odd segment
    int64_t launches = 0;
    for (int64_t sidx = 0; sidx < nseg; ++sidx) {
        const int64_t len = std::min<int64_t>((sidx + 1) * every, nsteps) - sidx * every;
        launches += len / 2 + len % 2;
    }
    if ((rc = adj_cuda(cudaMemsetAsync(d_galpha, 0, n * sizeof(double), st), err, errlen))) return rc;
    // lambda ping-pong between d_lam0 and d_lamwork, arranged so that lambda_0
    // lands in d_lam0
    double* lam = launches % 2 == 0 ? d_lam0 : d_lamwork;
    if ((rc = adj_cuda(cudaMemcpyAsync(lam, d_lamT, n * sizeof(double), cudaMemcpyDeviceToDevice, st),
                       err, errlen)))
        return rc;
    for (int64_t sidx = nseg - 1; sidx >= 0; --sidx) {
        const int64_t n0 = sidx * every, len = std::min<int64_t>(n0 + every, nsteps) - n0;
        // states u_{n0} .. u_{n0+len-1} of this segment
        const double* ck = d_checkpoints + (size_t)sidx * n;
        if ((rc = adj_cuda(cudaMemcpyAsync(d_states, ck, n * sizeof(double), cudaMemcpyDeviceToDevice,
                                           st), err, errlen)))
            return rc;
        int64_t j = 1;
        for (; j + 1 < len; j += 2)
            heatvar_step2<false><<<grid, 256, kStep2Smem, st>>>(d_states + (size_t)(j - 1) * n, d_courant,
                                                d_states + (size_t)j * n,
                                                d_states + (size_t)(j + 1) * n, nx, ny, rows);
        if (j < len)
            heatvar_step<false><<<grid_1, 256, kStepSmem, st>>>(d_states + (size_t)(j - 1) * n, d_courant,
                                                         d_states + (size_t)j * n, nx, ny, rows_1);
        // adjoint levels k = len-1 .. 0 of the segment (lambda_{n0+k+1} -> lambda_{n0+k})
        int64_t k = len - 1;
        for (; k >= 1; k -= 2) {
            double* out = lam == d_lam0 ? d_lamwork : d_lam0;
            heatvar_adjoint2<<<grid_a, 256, kAdj2Smem, st>>>(lam, d_courant, d_states + (size_t)k * n,
                                                     d_states + (size_t)(k - 1) * n, out,
                                                     d_galpha, nx, ny, rows_a);
            lam = out;
        }
        if (k == 0) {
            double* out = lam == d_lam0 ? d_lamwork : d_lam0;
            heatvar_adjoint<<<grid_1, 256, kAdjSmem, st>>>(lam, d_courant, d_states, out, d_galpha,
                                                           nx, ny, rows_1);
            lam = out;
        }
    }
    scale_kernel<<<1024, 256, 0, st>>>(d_galpha, n, dt / dx / dx);
    return adj_cuda(cudaGetLastError(), err, errlen);
}
