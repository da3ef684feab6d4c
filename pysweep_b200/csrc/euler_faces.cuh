// Euler with shared faces, standard decomposition: every face flux and every
// pressure of a level is evaluated once (the per-cell step evaluates each face
// twice, once from each of its cells, and each pressure ten times).  The
// arithmetic of every face and cell is that of Euler::step (euler::face,
// euler::dface, euler::update), so the results are bitwise equal.
#pragma once
#include "equations.cuh"
#include "swept.cuh"

namespace psb {

// 15 x 32 tiles: 512 faces between rows and 495 between columns, so each
// of the 256 threads takes at most two of each kind (no partial third pass
// at the barriers).
constexpr int kEuTR = 15, kEuTC = 32;                // tile rows, columns
constexpr int kEuHR = kEuTR + 4, kEuHC = kEuTC + 4;  // with the 2-cell halo
constexpr int kEuHRC = kEuHR * kEuHC;
constexpr int kEuXF = (kEuTR + 1) * kEuTC;  // faces between rows
constexpr int kEuYF = kEuTR * (kEuTC + 1);  // faces between columns
constexpr int kEuNT = 256;
static_assert(kEuXF <= 2 * kEuNT && kEuYF <= 2 * kEuNT && kEuTR * kEuTC <= 2 * kEuNT,
              "two faces and two cells per thread");
constexpr size_t kEuStdSmem = sizeof(double) * (4 * kEuHRC + kEuHRC + 8 * kEuXF + 8 * kEuYF);

__device__ __forceinline__ int eu_wrap(int v, int n)
{
    v %= n;
    return v < 0 ? v + n : v;
}

// Face e between rows (DIR 1: between halo rows j+1 and j+2, the lower face
// of tile row j) or between columns (DIR 2: between halo columns c+1 and
// c+2, the left face of tile column c) into f[0..7].
template <int DIR>
__device__ __forceinline__ void eu_face(const double* q, const double* P, int e, double gamma,
                                        double gm1, double* f)
{
    int ia, step;
    if (DIR == 1) {
        ia = (e / kEuTC + 1) * kEuHC + e % kEuTC + 2;
        step = kEuHC;
    } else {
        ia = (e / (kEuTC + 1) + 2) * kEuHC + e % (kEuTC + 1) + 1;
        step = 1;
    }
    const int ib = ia + step;
    double qa[4], qb[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        qa[v] = q[v * kEuHRC + ia];
        qb[v] = q[v * kEuHRC + ib];
    }
    euler::face<DIR>(gamma, gm1, qa, qb, P[ia - step], P[ia], P[ib], P[ib + step], f, f + 4);
}

// Two faces of one direction per thread, evaluated side by side (the second
// index is clamped and its result dropped where it lies past the last face).
template <int DIR, int NF>
__device__ __forceinline__ void eu_face_pair(const double* q, const double* P, double* F,
                                             int tid, double gamma, double gm1)
{
    const int e0 = tid, e1 = tid + kEuNT;
    const int e1c = e1 < NF ? e1 : NF - 1;
    double f0[8], f1[8];
    eu_face<DIR>(q, P, e0, gamma, gm1, f0);
    eu_face<DIR>(q, P, e1c, gamma, gm1, f1);
    if (e0 < NF) {
#pragma unroll
        for (int k = 0; k < 8; ++k) F[e0 * 8 + k] = f0[k];
    }
    if (e1 < NF) {
#pragma unroll
        for (int k = 0; k < 8; ++k) F[e1 * 8 + k] = f1[k];
    }
}

// One level for a 15 x 32 tile: the tile and its periodic halo into shared
// memory, the pressures, all faces (between rows and between columns, two
// of each per thread), then the stage update of every cell.
__global__ void __launch_bounds__(kEuNT, 2)
    euler_standard_faces(const double* __restrict__ cur, const double* __restrict__ prev,
                         double* __restrict__ out, double* __restrict__ frame, int nx, int ny,
                         int gts, EqParams p)
{
    extern __shared__ double sm[];
    double* q = sm;               // [4][HR][HC]
    double* P = q + 4 * kEuHRC;   // [HR][HC]
    double* FX = P + kEuHRC;      // [faces between rows][8]: flux 0..3, spectral 4..7
    double* FY = FX + 8 * kEuXF;  // [faces between columns][8]
    const int x0 = blockIdx.y * kEuTR, y0 = blockIdx.x * kEuTC;
    const int tid = threadIdx.x;
    const size_t plane = (size_t)nx * ny;
    const double dtdx = p.d[0], dtdy = p.d[1], gamma = p.d[2], gm1 = p.d[3];
    // the tile and its halo arrive by cp.async: every copy of a thread is in
    // flight at once
    for (int e = tid; e < 4 * kEuHRC; e += kEuNT) {
        const int c = e % kEuHC, r = (e / kEuHC) % kEuHR, v = e / kEuHRC;
        const int x = eu_wrap(x0 + r - 2, nx), y = eu_wrap(y0 + c - 2, ny);
        cp_async8(q + e, cur + v * plane + (size_t)x * ny + y);
    }
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
    for (int e = tid; e < kEuHRC; e += kEuNT)
        P[e] = euler::pressure(gm1, q[e], q[e + kEuHRC], q[e + 2 * kEuHRC], q[e + 3 * kEuHRC]);
    __syncthreads();
    eu_face_pair<1, kEuXF>(q, P, FX, tid, gamma, gm1);
    eu_face_pair<2, kEuYF>(q, P, FY, tid, gamma, gm1);
    __syncthreads();
    const bool full = gts % 2 == 0;
    for (int e = tid; e < kEuTR * kEuTC; e += kEuNT) {
        const int c = e % kEuTC, i = e / kEuTC;
        const int x = x0 + i, y = y0 + c;
        if (x >= nx || y >= ny) continue;
        const double* xlo = FX + (i * kEuTC + c) * 8;
        const double* xhi = xlo + kEuTC * 8;
        const double* ylo = FY + (i * (kEuTC + 1) + c) * 8;
        const double* yhi = ylo + 8;
        const size_t g = (size_t)x * ny + y;
        const int h = (i + 2) * kEuHC + c + 2;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const double o =
                euler::update(q[v * kEuHRC + h], full ? prev[v * plane + g] : 0.0,
                              euler::dface(xlo, xhi, v), euler::dface(ylo, yhi, v), dtdx, dtdy,
                              full);
            out[v * plane + g] = o;
            if (frame) frame[v * plane + g] = o;
        }
    }
}

}  // namespace psb
