// Standard decomposition for the heat equation (one variable): one level per
// launch, streaming rows (pysweep/core/pysweep.cu:259-275 computes the same
// step with one thread per cell and padded halos).
//
// A warp owns a 64-column strip and RB consecutive rows; lane l holds columns
// 2l, 2l+1.  Rows are streamed top to bottom with the rows above, at and
// below the centre in registers, so every value of the level is read from
// HBM once (plus one halo row above and below each RB-row strip and one halo
// column on each side for lanes 0 and 31).  The left / right neighbours come
// from the adjacent lanes by shuffle.  Arithmetic: Heat in equations.cuh.
// T is the storage type (double, or float with every level evaluated in
// double and rounded to float, as the reference's float32 runs do).
#pragma once
#include "heat_fast.cuh"

namespace psb {

constexpr int kStdRows = 32;  // rows per warp

template <bool RK2, class T = double>
__global__ void __launch_bounds__(256) heat_standard_fast(const T* __restrict__ cur,
                                                          const T* __restrict__ prev,
                                                          T* __restrict__ out,
                                                          T* __restrict__ frame, int nx,
                                                          int ny, int gts, double cr)
{
    using P = typename Pair2<T>::type;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int chunk = blockIdx.x * 8 + warp;
    const int cw = chunk * 64;
    if (cw >= ny) return;  // whole warp
    const int x0 = blockIdx.y * kStdRows;
    const int xend = min(x0 + kStdRows, nx);
    const int g = cw + 2 * lane;
    const int gl = cw == 0 ? ny - 1 : cw - 1;         // halo column left of the strip
    const int gr = cw + 64 == ny ? 0 : cw + 64;       // and right of it
    const int hcol = lane == 0 ? gl : gr;              // used by lanes 0 and 31
    auto row = [&](int x) -> const T* {
        x += x < 0 ? nx : 0;
        x -= x >= nx ? nx : 0;
        return cur + (size_t)x * ny;
    };
    double2 up = widen(*reinterpret_cast<const P*>(row(x0 - 1) + g));
    const T* rc = row(x0);
    double2 ce = widen(*reinterpret_cast<const P*>(rc + g));
    double hc = (lane == 0 || lane == 31) ? (double)rc[hcol] : 0.0;
    const bool full = (gts % 2 == 0);
    for (int x = x0; x < xend; ++x) {
        const T* rd = row(x + 1);
        const double2 dn = widen(*reinterpret_cast<const P*>(rd + g));
        const double hd = (lane == 0 || lane == 31) ? (double)rd[hcol] : 0.0;
        double left = __shfl_up_sync(0xffffffffu, ce.y, 1);
        double right = __shfl_down_sync(0xffffffffu, ce.x, 1);
        if (lane == 0) left = hc;
        if (lane == 31) right = hc;
        double n0, n1;
        if (!RK2) {
            n0 = to_level<T>(heat_fe(ce.x, up.x, dn.x, left, ce.y, cr));
            n1 = to_level<T>(heat_fe(ce.y, up.y, dn.y, ce.x, right, cr));
        } else {
            // heat.py:53-57: coeff*cd + base, base = u[t-1] on full steps
            const double cd0 = __dadd_rn(__dmul_rn(cr, __dadd_rn(__fma_rn(-2.0, ce.x, dn.x), up.x)),
                                         __dmul_rn(cr, __dadd_rn(__fma_rn(-2.0, ce.x, ce.y), left)));
            const double cd1 = __dadd_rn(__dmul_rn(cr, __dadd_rn(__fma_rn(-2.0, ce.y, dn.y), up.y)),
                                         __dmul_rn(cr, __dadd_rn(__fma_rn(-2.0, ce.y, right), ce.x)));
            double b0 = ce.x, b1 = ce.y;
            if (full) {
                const double2 pv = widen(*reinterpret_cast<const P*>(prev + (size_t)x * ny + g));
                b0 = pv.x;
                b1 = pv.y;
            }
            const double cf = full ? 1.0 : 0.5;
            n0 = to_level<T>(__dadd_rn(__dmul_rn(cf, cd0), b0));
            n1 = to_level<T>(__dadd_rn(__dmul_rn(cf, cd1), b1));
        }
        const size_t o = (size_t)x * ny + g;
        *reinterpret_cast<P*>(out + o) = pair2<T>(n0, n1);
        if (frame) *reinterpret_cast<P*>(frame + o) = pair2<T>(n0, n1);
        up = ce;
        ce = dn;
        hc = hd;
    }
}

}  // namespace psb
