// Built-in per-cell update functions ("step hooks") for the swept and
// standard engines.
//
// Each functor has the shape of the reference's GPU hook
//   __device__ void step(double* state, int idx, int globalTimeStep)
// (pysweep/core/pysweep.cu:25, pysweep/equations/heat.cu:35-48): it reads the
// current level around one cell and the level before it (for the Runge-Kutta
// roll-back), and writes the next level of that cell.  Because the swept engine
// keeps only a ring of levels in shared memory, the three levels are passed as
// three pointers instead of one pointer plus a TIMES stride; neighbours are at
// fixed element offsets (Nbr), like idx +- SY and idx +- 1 in the reference.
//
// Arithmetic follows the numpy CPU plugins operation by operation so that the
// GPU result is bitwise the CPU oracle's:
//   Heat     pysweep/equations/heat.py:21-31, :48-64
//   Euler    pysweep/equations/euler.py:131-313 (x**2 evaluated as x*x)
//   Example  pysweep/equations/example.py:13-26
//   Checker  pysweep/equations/checker.py:13-33
//   Half     pysweep/equations/half.py:15-19, :35-39
// The library is compiled with --fmad=false; fma() appears only where it is
// exactly equal to the separately rounded expression (a - 2*c: 2*c is exact).
#pragma once
#ifndef __CUDACC_RTC__  // run-time compilation (user step hooks) has no host headers
#include <cuda_runtime.h>
#endif

namespace psb {

struct EqParams {
    double d[8];
    int i[4];
    // grid fields read (and written) by equations that address cells by their
    // coordinates (variable diffusivity and its adjoint); fs = elements of one
    // level of f[1]
    double* f[3];
    long long fs;
};

// Element offsets of the points at distance k-2 along x (rows) and y (columns).
struct Nbr {
    int x[5];
    int y[5];
    int vs;  // variable stride
};

enum EqId {
    EQ_HEAT = 0,
    EQ_EULER = 1,
    EQ_EXAMPLE = 2,
    EQ_CHECKER = 3,
    EQ_HALF = 4,
    EQ_HEATVAR = 6,
    EQ_HEATVAR_ADJ = 7,
    EQ_HEATVAR_ADJMU = 8
};

// Equations whose step needs the cell's grid coordinates (Eq::kCoords and
// Eq::step_at(..., row, col)) instead of the tile pointers alone.
template <class Eq, class = void>
struct Coords {
    static constexpr bool value = false;
};
template <class Eq>
struct Coords<Eq, decltype((void)Eq::kCoords)> {
    static constexpr bool value = Eq::kCoords;
};

// heat.py: d[0] = courant = alpha*dt/dx/dx, i[0] = scheme (1 forward Euler, 0 RK2)
struct Heat {
    static constexpr int OPS = 1;
    static constexpr int ID = EQ_HEAT;
    __device__ static __forceinline__ void step(const double* __restrict__ u,
                                                const double* __restrict__ up,
                                                double* __restrict__ o, const Nbr& n, int gts,
                                                int nv, const EqParams& p)
    {
        const double c = u[0];
        const double cr = p.d[0];
        const double dxx = __dmul_rn(cr, __dadd_rn(__fma_rn(-2.0, c, u[n.x[3]]), u[n.x[1]]));
        const double dyy = __dmul_rn(cr, __dadd_rn(__fma_rn(-2.0, c, u[n.y[3]]), u[n.y[1]]));
        const double cd = __dadd_rn(dxx, dyy);
        if (p.i[0]) {
            o[0] = __dadd_rn(cd, c);
        } else {
            const bool full = (gts % 2 == 0);
            o[0] = __dadd_rn(__dmul_rn(full ? 1.0 : 0.5, cd), full ? up[0] : c);
        }
    }
};

// Heat, forward Euler, on float32 fields: the reference run with
// `dtype: float32` (pysweep/core/io.py:72-73) stores every level in float32,
// while heat.py's courant is a float64 scalar, so numpy evaluates the step in
// float64 (the order above) and rounds the result to float32 on store.
struct HeatF32 {
    static constexpr int OPS = 1;
    static constexpr int ID = EQ_HEAT;
    __device__ static __forceinline__ void step(const float* __restrict__ u,
                                                const float* __restrict__ up,
                                                float* __restrict__ o, const Nbr& n, int gts,
                                                int nv, const EqParams& p)
    {
        const double c = u[0];
        const double cr = p.d[0];
        const double dxx = __dmul_rn(cr, __dadd_rn(__fma_rn(-2.0, c, (double)u[n.x[3]]),
                                                   (double)u[n.x[1]]));
        const double dyy = __dmul_rn(cr, __dadd_rn(__fma_rn(-2.0, c, (double)u[n.y[3]]),
                                                   (double)u[n.y[1]]));
        o[0] = __double2float_rn(__dadd_rn(__dadd_rn(dxx, dyy), c));
    }
};

// half.py: (u[x+1]-2u+u[x-1])/100 + (u[y+1]-2u+u[y-1])/100, RK2 on gts%2
struct Half {
    static constexpr int OPS = 1;
    static constexpr int ID = EQ_HALF;
    __device__ static __forceinline__ void step(const double* __restrict__ u,
                                                const double* __restrict__ up,
                                                double* __restrict__ o, const Nbr& n, int gts,
                                                int nv, const EqParams& p)
    {
        const double c = u[0];
        const double a = __ddiv_rn(__dadd_rn(__fma_rn(-2.0, c, u[n.x[3]]), u[n.x[1]]), 100.0);
        const double b = __ddiv_rn(__dadd_rn(__fma_rn(-2.0, c, u[n.y[3]]), u[n.y[1]]), 100.0);
        const bool full = (gts % 2 == 0);
        o[0] = __dadd_rn(full ? up[0] : c, __dmul_rn(full ? 1.0 : 0.5, __dadd_rn(a, b)));
    }
};

// example.py: i[0] = scheme; forward: u+1; RK2: u[t-tc] + (2 or 1)
template <int OPS_>
struct ExampleT {
    static constexpr int OPS = OPS_;
    static constexpr int ID = EQ_EXAMPLE;
    __device__ static __forceinline__ void step(const double* __restrict__ u,
                                                const double* __restrict__ up,
                                                double* __restrict__ o, const Nbr& n, int gts,
                                                int nv, const EqParams& p)
    {
        for (int v = 0; v < nv; ++v) {
            const int q = v * n.vs;
            if (p.i[0]) {
                o[q] = __dadd_rn(u[q], 1.0);
            } else {
                const bool full = (gts % 2 == 0);
                o[q] = __dadd_rn(full ? up[q] : u[q], full ? 2.0 : 1.0);
            }
        }
    }
};

// checker.py: (((u[x+1] + u[x-1]) + u[y+1]) + u[y-1]) / 4
template <int OPS_>
struct CheckerT {
    static constexpr int OPS = OPS_;
    static constexpr int ID = EQ_CHECKER;
    __device__ static __forceinline__ void step(const double* __restrict__ u,
                                                const double* __restrict__ up,
                                                double* __restrict__ o, const Nbr& n, int gts,
                                                int nv, const EqParams& p)
    {
        for (int v = 0; v < nv; ++v) {
            const int q = v * n.vs;
            double s = __dadd_rn(u[q + n.x[3]], u[q + n.x[1]]);
            s = __dadd_rn(s, u[q + n.y[3]]);
            s = __dadd_rn(s, u[q + n.y[1]]);
            o[q] = __ddiv_rn(s, 4.0);
        }
    }
};

// ------------------------------------------------------------------ Euler --
// euler.py: d[0] = dtdx, d[1] = dtdy, d[2] = gamma, d[3] = gamma - 1
namespace euler {

__device__ __forceinline__ double pressure(double gm1, double q0, double q1, double q2, double q3)
{
    // euler.py:293  gM1*(q[3]-(q[1]*q[1]+q[2]*q[2])/(2*q[0]))
    return __dmul_rn(gm1, __dsub_rn(q3, __ddiv_rn(__dadd_rn(__dmul_rn(q1, q1), __dmul_rn(q2, q2)),
                                                  __dmul_rn(2.0, q0))));
}

// euler.py:250-256
__device__ __forceinline__ void limiter(const double* s1, const double* s2, double num, double den,
                                        double* out)
{
    double pr = __ddiv_rn(num, den);
    if (isnan(pr) || isinf(pr) || pr > 1e6 || pr < 0.0) pr = 0.0;
    const double h = __dmul_rn(1.0 < pr ? 1.0 : pr, 0.5);  // min(Pr,1)/2, exact halving
#pragma unroll
    for (int v = 0; v < 4; ++v) out[v] = __dadd_rn(s1[v], __dmul_rn(h, __dsub_rn(s2[v], s1[v])));
}

// evaluateFluxInX / evaluateFluxInY (euler.py:181-241); DIR 1 = x, 2 = y
template <int DIR>
__device__ __forceinline__ void flux(double gm1, const double* L, const double* R, double* f)
{
    const double pl = pressure(gm1, L[0], L[1], L[2], L[3]);
    const double pr = pressure(gm1, R[0], R[1], R[2], R[3]);
    constexpr int A = DIR;          // normal momentum component
    constexpr int B = 3 - DIR;      // tangential momentum component
    f[0] = __dadd_rn(L[A], R[A]);
    const double nn = __dadd_rn(__dadd_rn(__dadd_rn(__ddiv_rn(__dmul_rn(L[A], L[A]), L[0]), pl),
                                          __ddiv_rn(__dmul_rn(R[A], R[A]), R[0])),
                                pr);
    const double nt = __dadd_rn(__ddiv_rn(__dmul_rn(L[1], L[2]), L[0]),
                                __ddiv_rn(__dmul_rn(R[1], R[2]), R[0]));
    f[A] = nn;
    f[B] = nt;
    f[3] = __dadd_rn(__ddiv_rn(__dmul_rn(__dadd_rn(L[3], pl), L[A]), L[0]),
                     __ddiv_rn(__dmul_rn(__dadd_rn(R[3], pr), R[A]), R[0]));
}

// evaluateSpectral (euler.py:258-282)
template <int DIR>
__device__ __forceinline__ void spectral(double gamma, double gm1, const double* L,
                                         const double* R, double* s)
{
    const double rl = __dsqrt_rn(L[0]), rr = __dsqrt_rn(R[0]);
    const double denom = __ddiv_rn(1.0, __dadd_rn(rl, rr));
    double sp[4];
    sp[0] = __dmul_rn(rl, rr);
#pragma unroll
    for (int v = 1; v < 4; ++v) {
        const double tl = __ddiv_rn(L[v], L[0]);
        const double tr = __ddiv_rn(R[v], R[0]);
        sp[v] = __dmul_rn(__dadd_rn(__dmul_rn(rl, tl), __dmul_rn(rr, tr)), denom);
    }
    const double p = pressure(gm1, sp[0], __dmul_rn(sp[0], sp[1]), __dmul_rn(sp[0], sp[2]),
                              __dmul_rn(sp[0], sp[3]));
    double rad = __dadd_rn(__dsqrt_rn(__ddiv_rn(__dmul_rn(gamma, p), sp[0])), fabs(sp[DIR]));
    if (isnan(rad)) rad = 0.0;
#pragma unroll
    for (int v = 0; v < 4; ++v) s[v] = __dmul_rn(rad, __dsub_rn(L[v], R[v]));
}

// getFluxInX / getFluxInY for one cell (euler.py:158-223): o[k] = offset of
// the point at distance k-2 along the direction.
template <int DIR>
__device__ __forceinline__ void dflux(double gamma, double gm1, const double* __restrict__ u,
                                      const int* o, int vs, double* out)
{
    double q[5][4], P[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
#pragma unroll
        for (int v = 0; v < 4; ++v) q[k][v] = u[o[k] + v * vs];
        P[k] = pressure(gm1, q[k][0], q[k][1], q[k][2], q[k][3]);
    }
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    double L[4], R[4], f[4], s[4];
    limiter(q[1], q[2], __dsub_rn(P[2], P[1]), __dsub_rn(P[1], P[0]), L);
    limiter(q[2], q[1], __dsub_rn(P[2], P[1]), __dsub_rn(P[3], P[2]), R);
    flux<DIR>(gm1, L, R, f);
    spectral<DIR>(gamma, gm1, L, R, s);
#pragma unroll
    for (int v = 0; v < 4; ++v) acc[v] = __dadd_rn(__dadd_rn(acc[v], f[v]), s[v]);
    limiter(q[2], q[3], __dsub_rn(P[3], P[2]), __dsub_rn(P[2], P[1]), L);
    limiter(q[3], q[2], __dsub_rn(P[3], P[2]), __dsub_rn(P[4], P[3]), R);
    flux<DIR>(gm1, L, R, f);
    spectral<DIR>(gamma, gm1, L, R, s);
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        acc[v] = __dsub_rn(__dsub_rn(acc[v], f[v]), s[v]);
        out[v] = __dmul_rn(acc[v], 0.5);
    }
}

// One face between cells a (lower index) and b = a+1 in direction DIR: its
// flux f and spectral term s from q at a and b and the pressures at a-1, a,
// b, b+1.  dflux evaluates exactly this (same operations, same arguments)
// twice for every face, as the upper face of cell a and the lower face of
// cell b; the face-sharing kernels evaluate it once.
template <int DIR>
__device__ __forceinline__ void face(double gamma, double gm1, const double* qa, const double* qb,
                                     double Pam, double Pa, double Pb, double Pbp, double* f,
                                     double* s)
{
    double L[4], R[4];
    const double dab = __dsub_rn(Pb, Pa);
    limiter(qa, qb, dab, __dsub_rn(Pa, Pam), L);
    limiter(qb, qa, dab, __dsub_rn(Pbp, Pb), R);
    flux<DIR>(gm1, L, R, f);
    spectral<DIR>(gamma, gm1, L, R, s);
}

// A cell's derivative term from its lower (lo) and upper (hi) faces, each
// [flux 0..3, spectral 4..7], in dflux's order.
__device__ __forceinline__ double dface(const double* lo, const double* hi, int v)
{
    return __dmul_rn(__dsub_rn(__dsub_rn(__dadd_rn(__dadd_rn(0.0, lo[v]), lo[4 + v]), hi[v]),
                               hi[4 + v]),
                     0.5);
}

// The stage update of Euler::step (euler.py:131-156)
__device__ __forceinline__ double update(double u, double up, double fx, double fy, double dtdx,
                                         double dtdy, bool full)
{
    const double d = __dadd_rn(__dmul_rn(fx, dtdx), __dmul_rn(fy, dtdy));
    return full ? __dadd_rn(up, d) : __dadd_rn(u, __dmul_rn(0.5, d));
}

}  // namespace euler

// Scratch of Euler::level for a tile of bx rows and chunk w (doubles):
// pressures [bx][w+4], faces [(bx-3)*(w+1)][8], x-direction terms [(bx-4)*w][4].
__host__ __device__ constexpr int euler_level_scratch(int bx, int w)
{
    return bx * (w + 4) + 8 * (bx - 3) * (w + 1) + 4 * (bx - 4) * w;
}

struct Euler {
    static constexpr int OPS = 2;
    static constexpr int ID = EQ_EULER;
    static constexpr bool kFaceLevel = true;  // stream tiles use level() below

    // One level of a stream tile with faces shared between cells: out[i][kc+2]
    // from cur around (i, kc) and prv[i][kc-2] (the offsets of Eq::step in
    // stream_body) for rows [rlo, rhi) and columns kc in [kc0, kc1) of
    // [4][bx][rs] tiles.  Every thread of the CTA calls it (it synchronises);
    // scratch holds euler_level_scratch(bx, rs - 4) doubles.
    template <int NT>
    __device__ static void level(const double* __restrict__ cur, const double* __restrict__ prv,
                                 double* __restrict__ out, int rlo, int rhi, int kc0, int kc1,
                                 int rs, int bx, int gts, const EqParams& p, double* scratch,
                                 int tid)
    {
        const int vs = bx * rs;
        const int nr = rhi - rlo, nc = kc1 - kc0;
        if (nr <= 0 || nc <= 0) return;  // the same for every thread
        const double dtdx = p.d[0], dtdy = p.d[1], gamma = p.d[2], gm1 = p.d[3];
        double* P = scratch;                      // [bx][rs]
        double* F = P + bx * rs;                  // faces, [.][8]
        double* D = F + 8 * (bx - 3) * (rs - 3);  // x terms, [nr][nc][4]
        const int pc = nc + 4, npr = (nr + 4) * pc;
        for (int e = tid; e < npr; e += NT) {
            const int o = (rlo - 2 + e / pc) * rs + kc0 - 2 + e % pc;
            P[o] = euler::pressure(gm1, cur[o], cur[o + vs], cur[o + 2 * vs], cur[o + 3 * vs]);
        }
        __syncthreads();
        // faces between rows rlo-1+j and rlo+j
        for (int e = tid; e < (nr + 1) * nc; e += NT) {
            const int a = (rlo - 1 + e / nc) * rs + kc0 + e % nc, b = a + rs;
            double qa[4], qb[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                qa[v] = cur[a + v * vs];
                qb[v] = cur[b + v * vs];
            }
            euler::face<1>(gamma, gm1, qa, qb, P[a - rs], P[a], P[b], P[b + rs], F + e * 8,
                           F + e * 8 + 4);
        }
        __syncthreads();
        for (int e = tid; e < nr * nc; e += NT) {
#pragma unroll
            for (int v = 0; v < 4; ++v) D[e * 4 + v] = euler::dface(F + e * 8, F + (e + nc) * 8, v);
        }
        __syncthreads();
        // faces between columns kc0-1+c and kc0+c
        for (int e = tid; e < nr * (nc + 1); e += NT) {
            const int a = (rlo + e / (nc + 1)) * rs + kc0 - 1 + e % (nc + 1), b = a + 1;
            double qa[4], qb[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                qa[v] = cur[a + v * vs];
                qb[v] = cur[b + v * vs];
            }
            euler::face<2>(gamma, gm1, qa, qb, P[a - 1], P[a], P[b], P[b + 1], F + e * 8,
                           F + e * 8 + 4);
        }
        __syncthreads();
        const bool full = gts % 2 == 0;
        for (int e = tid; e < nr * nc; e += NT) {
            const int i = e / nc, c = e % nc;
            const int o = (rlo + i) * rs + kc0 + c;
            const double* lo = F + (i * (nc + 1) + c) * 8;
#pragma unroll
            for (int v = 0; v < 4; ++v)
                out[o + OPS + v * vs] =
                    euler::update(cur[o + v * vs], prv[o - OPS + v * vs], D[e * 4 + v],
                                  euler::dface(lo, lo + 8, v), dtdx, dtdy, full);
        }
    }

    __device__ static __forceinline__ void step(const double* __restrict__ u,
                                                const double* __restrict__ up,
                                                double* __restrict__ o, const Nbr& n, int gts,
                                                int nv, const EqParams& p)
    {
        double fx[4], fy[4];
        euler::dflux<1>(p.d[2], p.d[3], u, n.x, n.vs, fx);
        euler::dflux<2>(p.d[2], p.d[3], u, n.y, n.vs, fy);
        const double dtdx = p.d[0], dtdy = p.d[1];
        if (gts % 2 == 0) {
#pragma unroll
            for (int v = 0; v < 4; ++v)
                o[v * n.vs] = __dadd_rn(up[v * n.vs],
                                        __dadd_rn(__dmul_rn(fx[v], dtdx), __dmul_rn(fy[v], dtdy)));
        } else {
#pragma unroll
            for (int v = 0; v < 4; ++v)
                o[v * n.vs] = __dadd_rn(
                    u[v * n.vs],
                    __dmul_rn(0.5, __dadd_rn(__dmul_rn(fx[v], dtdx), __dmul_rn(fy[v], dtdy))));
        }
    }
};

// Euler with the per-cell step in the stream tiles too (blocksizes whose
// tile leaves no room for the face scratch)
struct EulerCell : Euler {
    static constexpr bool kFaceLevel = false;
};

// Heat with a courant number per cell, C = f[0][row][col] (the
// differentiable solve's forward step, heatvar_step in adjoint.cu):
//     u' = (C*((u[x+1]-2u)+u[x-1]) + C*((u[y+1]-2u)+u[y-1])) + u,
// the heat plugin's order (pysweep/equations/heat.py:60-64) with the courant
// number per cell.  With f[1] set, the step also stores the old level's
// Laplacian ((u[x+1]-2u)+u[x-1]) + ((u[y+1]-2u)+u[y-1]) at
// f[1][(gts-1)*fs + row*ny + col]: the recompute of one checkpoint segment for
// the adjoint.  i[1] = nx, i[2] = ny.
struct HeatVar {
    static constexpr int OPS = 1;
    static constexpr int ID = EQ_HEATVAR;
    static constexpr bool kCoords = true;
    __device__ static __forceinline__ void step_at(const double* __restrict__ u,
                                                   const double* __restrict__, double* __restrict__ o,
                                                   const Nbr& n, int gts, int, const EqParams& p,
                                                   int row, int col)
    {
        const size_t at = (size_t)row * p.i[2] + col;
        const double c = u[0];
        const double C = __ldg(p.f[0] + at);
        const double rx = __dadd_rn(__fma_rn(-2.0, c, u[n.x[3]]), u[n.x[1]]);
        const double ry = __dadd_rn(__fma_rn(-2.0, c, u[n.y[3]]), u[n.y[1]]);
        o[0] = __dadd_rn(__dadd_rn(__dmul_rn(C, rx), __dmul_rn(C, ry)), c);
        if (p.f[1]) p.f[1][(size_t)(gts - 1) * p.fs + at] = __dadd_rn(rx, ry);
    }
};

// The adjoint of HeatVar (heatvar_adjoint in adjoint.cu), run backward in
// time through one checkpoint segment of i[3] steps.  Variable 0 is lambda,
// variable 1 the accumulated dJ/dC.  Level gts (1-based in the segment) takes
// lambda_{n+1} to
//     lambda_n = lambda_{n+1} + L(C .* lambda_{n+1})
// (L the periodic 5-point Laplacian in the order above, C .* lambda formed at
// each of the five cells) and adds lambda_{n+1} * L(u_n) to dJ/dC in one fused
// multiply-add, n = segment end - gts, L(u_n) from the segment's recompute at
// f[1][(i[3]-gts)*fs + row*ny + col].  Each cell's levels are evaluated in
// order in every decomposition, so dJ/dC sums in the same order as the
// standard adjoint kernels.  i[1] = nx, i[2] = ny.
struct HeatVarAdj {
    static constexpr int OPS = 1;
    static constexpr int ID = EQ_HEATVAR_ADJ;
    static constexpr bool kCoords = true;
    __device__ static __forceinline__ void step_at(const double* __restrict__ u,
                                                   const double* __restrict__, double* __restrict__ o,
                                                   const Nbr& n, int gts, int, const EqParams& p,
                                                   int row, int col)
    {
        const int nx = p.i[1], ny = p.i[2];
        const double* C = p.f[0];
        const int rm = row == 0 ? nx - 1 : row - 1, rp = row + 1 == nx ? 0 : row + 1;
        const int cm = col == 0 ? ny - 1 : col - 1, cp = col + 1 == ny ? 0 : col + 1;
        const size_t at = (size_t)row * ny + col;
        const double l = u[0];
        const double mc = __dmul_rn(__ldg(C + at), l);
        const double mxp = __dmul_rn(__ldg(C + (size_t)rp * ny + col), u[n.x[3]]);
        const double mxm = __dmul_rn(__ldg(C + (size_t)rm * ny + col), u[n.x[1]]);
        const double myp = __dmul_rn(__ldg(C + (size_t)row * ny + cp), u[n.y[3]]);
        const double mym = __dmul_rn(__ldg(C + (size_t)row * ny + cm), u[n.y[1]]);
        const double lm = __dadd_rn(__dadd_rn(__fma_rn(-2.0, mc, mxp), mxm),
                                    __dadd_rn(__fma_rn(-2.0, mc, myp), mym));
        o[0] = __dadd_rn(l, lm);
        const double lu = __ldg(p.f[1] + (size_t)(p.i[3] - gts) * p.fs + at);
        o[n.vs] = __fma_rn(l, lu, u[n.vs]);
    }
};

// The adjoint of HeatVar in the variable mu = C .* lambda: with L symmetric,
// lambda_n = lambda_{n+1} + L(C .* lambda_{n+1}) is
//     mu_n = mu_{n+1} + C .* L(mu_{n+1}),
// HeatVar's own step (same operation order) applied to mu, and
// dJ/dC = sum_n lambda_{n+1} .* L(u_n) = (sum_n mu_{n+1} .* L(u_n)) ./ C.
// One variable (mu); level gts (1-based in a checkpoint segment of i[3] steps)
// reads L(u_n), n = segment end - gts, at f[1][(i[3]-gts)*fs + row*ny + col]
// and adds mu_{n+1} * L(u_n) to f[2][row*ny + col] in place (one fused
// multiply-add per cell and level, in level order in every decomposition).
// The register-resident streams (heat_fast.cuh, per-cell courant) do the
// same arithmetic.  i[1] = nx, i[2] = ny.
struct HeatVarAdjMu {
    static constexpr int OPS = 1;
    static constexpr int ID = EQ_HEATVAR_ADJMU;
    static constexpr bool kCoords = true;
    __device__ static __forceinline__ void step_at(const double* __restrict__ u,
                                                   const double* __restrict__, double* __restrict__ o,
                                                   const Nbr& n, int gts, int, const EqParams& p,
                                                   int row, int col)
    {
        const size_t at = (size_t)row * p.i[2] + col;
        const double c = u[0];
        const double C = __ldg(p.f[0] + at);
        const double rx = __dadd_rn(__fma_rn(-2.0, c, u[n.x[3]]), u[n.x[1]]);
        const double ry = __dadd_rn(__fma_rn(-2.0, c, u[n.y[3]]), u[n.y[1]]);
        o[0] = __dadd_rn(__dadd_rn(__dmul_rn(C, rx), __dmul_rn(C, ry)), c);
        const double lu = __ldg(p.f[1] + (size_t)(p.i[3] - gts) * p.fs + at);
        p.f[2][at] = __fma_rn(c, lu, p.f[2][at]);
    }
};

}  // namespace psb
