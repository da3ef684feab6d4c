// Euler with shared faces, standard decomposition: every face flux and every
// pressure of a level is evaluated once (the per-cell step evaluates each face
// twice, once from each of its cells, and each pressure ten times).  The
// arithmetic of every face and cell is that of Euler::step (euler::face,
// euler::dface, euler::update), so the results are bitwise equal.
#pragma once
#include "equations.cuh"

namespace psb {

constexpr int kEuTR = 16, kEuTC = 32;                // tile rows, columns
constexpr int kEuHR = kEuTR + 4, kEuHC = kEuTC + 4;  // with the 2-cell halo
constexpr int kEuHRC = kEuHR * kEuHC;
constexpr int kEuXF = (kEuTR + 1) * kEuTC;  // faces between rows
constexpr int kEuYF = kEuTR * (kEuTC + 1);  // faces between columns
constexpr int kEuF = kEuXF > kEuYF ? kEuXF : kEuYF;
constexpr size_t kEuStdSmem = sizeof(double) * (4 * kEuHRC + kEuHRC + 8 * kEuF + 4 * kEuTR * kEuTC);

__device__ __forceinline__ int eu_wrap(int v, int n)
{
    v %= n;
    return v < 0 ? v + n : v;
}

// One level for a 16 x 32 tile: the tile and its periodic halo into shared
// memory, the pressures, the faces between rows (x-direction terms per
// cell), the faces between columns, then the stage update.
__global__ void __launch_bounds__(256, 2)
    euler_standard_faces(const double* __restrict__ cur, const double* __restrict__ prev,
                         double* __restrict__ out, double* __restrict__ frame, int nx, int ny,
                         int gts, EqParams p)
{
    extern __shared__ double sm[];
    double* q = sm;              // [4][HR][HC]
    double* P = q + 4 * kEuHRC;  // [HR][HC]
    double* F = P + kEuHRC;      // [faces][8]: flux 0..3, spectral 4..7
    double* D = F + 8 * kEuF;    // [TR][TC][4]: x-direction terms
    const int x0 = blockIdx.y * kEuTR, y0 = blockIdx.x * kEuTC;
    const int tid = threadIdx.x;
    const size_t plane = (size_t)nx * ny;
    const double dtdx = p.d[0], dtdy = p.d[1], gamma = p.d[2], gm1 = p.d[3];
    for (int e = tid; e < 4 * kEuHRC; e += 256) {
        const int c = e % kEuHC, r = (e / kEuHC) % kEuHR, v = e / kEuHRC;
        const int x = eu_wrap(x0 + r - 2, nx), y = eu_wrap(y0 + c - 2, ny);
        q[e] = cur[v * plane + (size_t)x * ny + y];
    }
    __syncthreads();
    for (int e = tid; e < kEuHRC; e += 256)
        P[e] = euler::pressure(gm1, q[e], q[e + kEuHRC], q[e + 2 * kEuHRC], q[e + 3 * kEuHRC]);
    __syncthreads();
    // faces between halo rows j+1 and j+2 (the lower face of tile row j)
    for (int e = tid; e < kEuXF; e += 256) {
        const int c = e % kEuTC, j = e / kEuTC;
        const int ia = (j + 1) * kEuHC + c + 2, ib = ia + kEuHC;
        double qa[4], qb[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            qa[v] = q[v * kEuHRC + ia];
            qb[v] = q[v * kEuHRC + ib];
        }
        euler::face<1>(gamma, gm1, qa, qb, P[ia - kEuHC], P[ia], P[ib], P[ib + kEuHC], F + e * 8,
                       F + e * 8 + 4);
    }
    __syncthreads();
    for (int e = tid; e < kEuTR * kEuTC; e += 256) {
        const int c = e % kEuTC, i = e / kEuTC;
        const double* lo = F + (i * kEuTC + c) * 8;
        const double* hi = lo + kEuTC * 8;
#pragma unroll
        for (int v = 0; v < 4; ++v) D[e * 4 + v] = euler::dface(lo, hi, v);
    }
    __syncthreads();
    // faces between halo columns c+1 and c+2 (the left face of tile column c)
    for (int e = tid; e < kEuYF; e += 256) {
        const int c = e % (kEuTC + 1), i = e / (kEuTC + 1);
        const int ia = (i + 2) * kEuHC + c + 1, ib = ia + 1;
        double qa[4], qb[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            qa[v] = q[v * kEuHRC + ia];
            qb[v] = q[v * kEuHRC + ib];
        }
        euler::face<2>(gamma, gm1, qa, qb, P[ia - 1], P[ia], P[ib], P[ib + 1], F + e * 8,
                       F + e * 8 + 4);
    }
    __syncthreads();
    const bool full = gts % 2 == 0;
    for (int e = tid; e < kEuTR * kEuTC; e += 256) {
        const int c = e % kEuTC, i = e / kEuTC;
        const int x = x0 + i, y = y0 + c;
        if (x >= nx || y >= ny) continue;
        const double* lo = F + (i * (kEuTC + 1) + c) * 8;
        const double* hi = lo + 8;
        const size_t g = (size_t)x * ny + y;
        const int h = (i + 2) * kEuHC + c + 2;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const double o = euler::update(q[v * kEuHRC + h], full ? prev[v * plane + g] : 0.0,
                                           D[e * 4 + v], euler::dface(lo, hi, v), dtdx, dtdy, full);
            out[v * plane + g] = o;
            if (frame) frame[v * plane + g] = o;
        }
    }
}

}  // namespace psb
