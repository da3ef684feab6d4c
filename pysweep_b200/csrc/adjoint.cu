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
// through the segment; each adjoint step updates lambda and accumulates the
// gradient in one pass.
//
// All kernels stream 64-column strips down 32-row blocks: lane l holds columns
// 2l, 2l+1, the rows above/at/below in registers, lateral neighbours by
// shuffle (the layout of heat_standard_fast).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>

#include "../../include/pysweep_b200.h"
#include "heat_fast.cuh"

namespace psb {
namespace {

constexpr int kRows = 32;

struct Strip {
    int nx, ny, g, x0, xend, lane, hcol;
    __device__ Strip(int nx_, int ny_) : nx(nx_), ny(ny_)
    {
        const int warp = threadIdx.x >> 5;
        lane = threadIdx.x & 31;
        const int cw = (blockIdx.x * 8 + warp) * 64;
        g = cw + 2 * lane;
        x0 = blockIdx.y * kRows;
        xend = min(x0 + kRows, nx);
        const int gl = cw == 0 ? ny - 1 : cw - 1;
        const int gr = cw + 64 == ny ? 0 : cw + 64;
        hcol = lane == 0 ? gl : gr;
    }
    __device__ bool active() const { return g - 2 * lane < ny; }
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

__device__ __forceinline__ Row load_row(const double* f, const Strip& s, int x)
{
    const double* p = f + s.row(x);
    const double2 v = *reinterpret_cast<const double2*>(p + s.g);
    Row r;
    r.a = v.x;
    r.b = v.y;
    r.h = (s.lane == 0 || s.lane == 31) ? p[s.hcol] : 0.0;
    return r;
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

__global__ void courant_kernel(const double* __restrict__ alpha, double* __restrict__ C, size_t n,
                               double dt, double dx)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        C[i] = alpha[i] * dt / dx / dx;
}

// u' = (C*dxx + C*dyy) + u
__global__ void __launch_bounds__(256) heatvar_step(const double* __restrict__ u,
                                                    const double* __restrict__ C,
                                                    double* __restrict__ out, int nx, int ny)
{
    const Strip s(nx, ny);
    if (!s.active()) return;
    Row up = load_row(u, s, s.x0 - 1), ce = load_row(u, s, s.x0);
    for (int x = s.x0; x < s.xend; ++x) {
        const Row dn = load_row(u, s, x + 1);
        double left = __shfl_up_sync(0xffffffffu, ce.b, 1);
        double right = __shfl_down_sync(0xffffffffu, ce.a, 1);
        if (s.lane == 0) left = ce.h;
        if (s.lane == 31) right = ce.h;
        const size_t o = s.row(x) + s.g;
        const double2 cr = *reinterpret_cast<const double2*>(C + o);
        const double n0 = heat_fe(ce.a, up.a, dn.a, left, ce.b, cr.x);
        const double n1 = heat_fe(ce.b, up.b, dn.b, ce.a, right, cr.y);
        *reinterpret_cast<double2*>(out + o) = make_double2(n0, n1);
        up = ce;
        ce = dn;
    }
}

// One adjoint level: lam_out = lam + L(C .* lam);  gC += lam .* L(u)
__global__ void __launch_bounds__(256) heatvar_adjoint(const double* __restrict__ lam,
                                                       const double* __restrict__ C,
                                                       const double* __restrict__ u,
                                                       double* __restrict__ lam_out,
                                                       double* __restrict__ gC, int nx, int ny)
{
    const Strip s(nx, ny);
    if (!s.active()) return;
    auto mu_row = [&](int x) {
        const Row l = load_row(lam, s, x), c = load_row(C, s, x);
        Row m;
        m.a = __dmul_rn(c.a, l.a);
        m.b = __dmul_rn(c.b, l.b);
        m.h = __dmul_rn(c.h, l.h);
        return m;
    };
    Row mup = mu_row(s.x0 - 1), mce = mu_row(s.x0);
    Row uup = load_row(u, s, s.x0 - 1), uce = load_row(u, s, s.x0);
    for (int x = s.x0; x < s.xend; ++x) {
        const Row mdn = mu_row(x + 1), udn = load_row(u, s, x + 1);
        double lm0, lm1, lu0, lu1;
        lap(mup, mce, mdn, s.lane, lm0, lm1);
        lap(uup, uce, udn, s.lane, lu0, lu1);
        const size_t o = s.row(x) + s.g;
        const double2 l = *reinterpret_cast<const double2*>(lam + o);
        const double2 gc = *reinterpret_cast<const double2*>(gC + o);
        *reinterpret_cast<double2*>(lam_out + o) = make_double2(__dadd_rn(l.x, lm0), __dadd_rn(l.y, lm1));
        *reinterpret_cast<double2*>(gC + o) =
            make_double2(__fma_rn(l.x, lu0, gc.x), __fma_rn(l.y, lu1, gc.y));
        mup = mce;
        mce = mdn;
        uup = uce;
        uce = udn;
    }
}

__global__ void scale_kernel(double* __restrict__ g, size_t n, double f)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        g[i] *= f;
}

dim3 strip_grid(int nx, int ny) { return dim3((ny / 64 + 7) / 8, (nx + kRows - 1) / kRows); }

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
        heatvar_step<<<strip_grid(nx, ny), 256, 0, st>>>(in, d_courant, out, nx, ny);
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
    const dim3 grid = strip_grid(nx, ny);
    if ((rc = adj_cuda(cudaMemsetAsync(d_galpha, 0, n * sizeof(double), st), err, errlen))) return rc;
    // lambda ping-pong: d_lam0 and d_lamwork, arranged so that lambda_0 lands in d_lam0
    if ((rc = adj_cuda(cudaMemcpyAsync(nsteps % 2 == 0 ? d_lam0 : d_lamwork, d_lamT, n * sizeof(double),
                                       cudaMemcpyDeviceToDevice, st), err, errlen)))
        return rc;
    double* lam = nsteps % 2 == 0 ? d_lam0 : d_lamwork;
    const int64_t nseg = (nsteps + every - 1) / every;
    for (int64_t sidx = nseg - 1; sidx >= 0; --sidx) {
        const int64_t n0 = sidx * every, n1 = std::min<int64_t>(n0 + every, nsteps);
        // states u_{n0} .. u_{n1-1} of this segment
        const double* ck = d_checkpoints + (size_t)sidx * n;
        if ((rc = adj_cuda(cudaMemcpyAsync(d_states, ck, n * sizeof(double), cudaMemcpyDeviceToDevice,
                                           st), err, errlen)))
            return rc;
        for (int64_t j = 1; j < n1 - n0; ++j)
            heatvar_step<<<grid, 256, 0, st>>>(d_states + (size_t)(j - 1) * n, d_courant,
                                               d_states + (size_t)j * n, nx, ny);
        for (int64_t nn = n1 - 1; nn >= n0; --nn) {
            double* out = lam == d_lam0 ? d_lamwork : d_lam0;
            heatvar_adjoint<<<grid, 256, 0, st>>>(lam, d_courant, d_states + (size_t)(nn - n0) * n, out,
                                                  d_galpha, nx, ny);
            lam = out;
        }
    }
    scale_kernel<<<1024, 256, 0, st>>>(d_galpha, n, dt / dx / dx);
    return adj_cuda(cudaGetLastError(), err, errlen);
}
