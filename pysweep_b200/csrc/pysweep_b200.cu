// C ABI of the B200 swept space-time solver (declarations: include/pysweep_b200.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <functional>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/pysweep_b200.h"
#include "equations.cuh"
#include "swept.cuh"
#include "heat_fast.cuh"
#include "seam_fast.cuh"
#include "standard_fast.cuh"
#include "euler_faces.cuh"
#include "batch.cuh"
#include "hook.cuh"

namespace psb {

// ---------------------------------------------------------- standard ------
// One level of the standard decomposition (pysweep/core/pysweep.cu:259-275,
// functions.py:126-146): every cell of level L+1 from levels L and L-1, with
// periodic neighbours taken directly instead of through padded halos.
template <class Eq>
__global__ void __launch_bounds__(256) standard_kernel(const double* __restrict__ cur,
                                                       const double* __restrict__ prev,
                                                       double* __restrict__ out,
                                                       double* __restrict__ frame, int nx, int ny,
                                                       int nv, int gts, EqParams p)
{
    const int y = blockIdx.x * blockDim.x + threadIdx.x;
    const int x = blockIdx.y;
    if (y >= ny) return;
    Nbr n;
    n.vs = nx * ny;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        int xx = x + k - 2, yy = y + k - 2;
        xx += xx < 0 ? nx : (xx >= nx ? -nx : 0);
        yy += yy < 0 ? ny : (yy >= ny ? -ny : 0);
        n.x[k] = (xx - x) * ny;
        n.y[k] = yy - y;
    }
    const size_t c = (size_t)x * ny + y;
    if constexpr (Coords<Eq>::value)
        Eq::step_at(cur + c, prev + c, out + c, n, gts, nv, p, x, y);
    else
        Eq::step(cur + c, prev + c, out + c, n, gts, nv, p);
    if (frame) {
        for (int v = 0; v < nv; ++v) frame[c + (size_t)v * n.vs] = out[c + (size_t)v * n.vs];
    }
}

}  // namespace psb

using namespace psb;

struct ps_solver {
    int device = 0;
    int eq = 0;
    int nv = 1, nx = 0, ny = 0, ops = 1, its = 1, bs = 0;
    int mpss = 0;
    int dtype = PS_DTYPE_F64;
    size_t esize = sizeof(double);  // bytes per element of every field and face buffer
    // tiling
    int H = 0, nseg = 1, chunk = 32, threads = 128;
    // heatvar / heatvar adjoint: courant numbers, the segment's recomputed
    // Laplacians (ps_set_field; device memory the caller owns)
    double* field[3] = {nullptr, nullptr, nullptr};
    bool nseg_auto = true;  // choose the segment count per run until configured
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    // the gap stream runs beside the y-bridge seam on a high-priority side
    // stream (forked from and joined back into `stream` with two events)
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    // named plugin constants
    std::map<std::string, double> globals;
    // device buffers
    double* base[2] = {nullptr, nullptr};  // [its][nv][nx][ny] each
    int cur = 0;                           // which base holds the current levels
    bool have_state = false;
    double* xface = nullptr;
    size_t xface_n = 0;
    double* yface = nullptr;
    size_t yface_n = 0;
    double* ring[3] = {nullptr, nullptr, nullptr};
    int64_t launches = 0;
    std::string err;
    // optional per-kernel device timing (ps_profile): events around every launch
    bool profile = false;
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> pending;
    std::vector<cudaEvent_t> event_pool;
    double prof_ms[8] = {0};
    int64_t prof_n[8] = {0};
    // algorithmic cell updates per kernel kind, accumulated with prof_ms
    double prof_cells[8] = {0};
    // user step hook compiled at run time (ps_create_hook); nullptr for the
    // built-in equations
    HookModule* hook = nullptr;
    std::string hook_src;    // the hook's source (declared types of its constants)
    std::string launch_err;  // a driver-API launch failure, reported by check_launch
};

namespace {

const char* kVersion = "pysweep_b200 0.1.0 (sm_100a)";
thread_local std::string g_create_error;  // message of the last failed ps_create

// Opt a kernel into the large dynamic shared-memory carve-out, once per
// (kernel, device).
std::mutex g_attr_mu;
std::map<std::pair<const void*, int>, bool> g_attr_done;

template <class K>
void allow_big_smem(K kernel)
{
    int dev = 0;
    cudaGetDevice(&dev);
    const auto key = std::make_pair(reinterpret_cast<const void*>(kernel), dev);
    std::lock_guard<std::mutex> lock(g_attr_mu);
    if (!g_attr_done[key]) {
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        g_attr_done[key] = true;
    }
}

int fail(ps_solver* s, int code, const char* fmt, ...)
{
    if (s) {
        va_list ap, ap2;
        va_start(ap, fmt);
        va_copy(ap2, ap);
        const int n = vsnprintf(nullptr, 0, fmt, ap);
        va_end(ap);
        std::string buf(n > 0 ? (size_t)n : 0, '\0');
        if (n > 0) vsnprintf(&buf[0], (size_t)n + 1, fmt, ap2);
        va_end(ap2);
        s->err = buf;  // any length: hook compiler logs included
    }
    return code;
}

#define PS_CUDA(s, call)                                                                       \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            return fail((s), e_ == cudaErrorMemoryAllocation ? PS_ERR_NOMEM : PS_ERR_CUDA,     \
                        "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

size_t field_elems(const ps_solver* s) { return (size_t)s->nv * s->nx * s->ny; }
// element offsets and sizes in the solver's storage type (double or float;
// device buffers are kept as double* and addressed in bytes)
double* at(const ps_solver* s, double* p, size_t elems)
{
    return reinterpret_cast<double*>(reinterpret_cast<char*>(p) + elems * s->esize);
}
size_t nbytes(const ps_solver* s, size_t elems) { return elems * s->esize; }

int eq_ops(int eq, int ops)
{
    switch (eq) {
    case PS_EQ_HEAT: return 1;
    case PS_EQ_HALF: return 1;
    case PS_EQ_HEATVAR: return 1;
    case PS_EQ_HEATVAR_ADJ: return 1;
    case PS_EQ_HEATVAR_ADJMU: return 1;
    case PS_EQ_EULER: return 2;
    default: return ops;  // example / checker take the configured ops
    }
}

// Equation constants, computed on the host the way each plugin's set_globals
// computes its CPU globals (heat.py:37, euler.py:23-24).
EqParams make_params_g(int eq, const std::map<std::string, double>& globals)
{
    EqParams p;
    memset(&p, 0, sizeof p);
    auto g = [&](const char* k, double d) {
        auto it = globals.find(k);
        return it == globals.end() ? d : it->second;
    };
    switch (eq) {
    case PS_EQ_HEAT: {
        const double alpha = g("ALPHA", 1.0), dt = g("DT", 0.0), dx = g("DX", 1.0);
        p.d[0] = alpha * dt / dx / dx;
        p.i[0] = g("SCHEME", 1.0) != 0.0;
        break;
    }
    case PS_EQ_EULER: {
        const double dt = g("DT", 0.0), dx = g("DX", 1.0), dy = g("DY", dx);
        const double gamma = g("GAMMA", 1.4);
        p.d[0] = g("DTDX", dt / dx);
        p.d[1] = g("DTDY", dt / dy);
        p.d[2] = gamma;
        p.d[3] = g("GAM_M1", gamma - 1.0);
        break;
    }
    case PS_EQ_EXAMPLE:
    case PS_EQ_CHECKER: p.i[0] = g("SCHEME", 1.0) != 0.0; break;
    default: break;
    }
    return p;
}

EqParams make_params(const ps_solver* s)
{
    EqParams p = make_params_g(s->eq, s->globals);
    if (s->eq == PS_EQ_HEATVAR || s->eq == PS_EQ_HEATVAR_ADJ || s->eq == PS_EQ_HEATVAR_ADJMU) {
        p.i[1] = s->nx;
        p.i[2] = s->ny;
        auto it = s->globals.find("LEN");
        p.i[3] = it == s->globals.end() ? 0 : (int)it->second;
        p.f[0] = s->field[0];
        p.f[1] = s->field[1];
        p.f[2] = s->field[2];
        p.fs = (long long)s->nx * s->ny;
    }
    return p;
}

// Equation id of solvers running a user step hook (internal: ps_create_hook)
constexpr int PS_EQ_HOOK = 5;

// ------------------------------------------------------------ dispatch ----
using SweptLaunch = std::function<void(const SweptArgs&, int grid, size_t smem, cudaStream_t)>;
using StdLaunch = void (*)(const double*, const double*, double*, double*, int, int, int, int,
                           const EqParams&, cudaStream_t);

template <class Eq, int ITS, int W, bool GAP>
void launch_stream(const SweptArgs& a, int grid, size_t smem, cudaStream_t st)
{
    auto k = stream_kernel<Eq, ITS, W, GAP, 256>;
    allow_big_smem(k);
    k<<<grid, 256, smem, st>>>(a);
}

template <class Eq, int ITS, bool GAP, class T = double>
void launch_seam(const SweptArgs& a, int grid, size_t smem, cudaStream_t st)
{
    // one-variable stencils: 64 threads per seam (the seams are issue-bound
    // on per-level loop work that every warp repeats; measured 1-2% faster
    // in total than 128); Euler keeps 128 for its four-variable tiles
    constexpr int NT = Eq::OPS == 1 ? 64 : 128;
    auto k = seam_kernel<Eq, ITS, GAP, NT, T>;
    allow_big_smem(k);
    k<<<grid, NT, smem, st>>>(a);
}

template <class Eq>
void launch_standard(const double* cur, const double* prev, double* out, double* frame, int nx,
                     int ny, int nv, int gts, const EqParams& p, cudaStream_t st)
{
    dim3 grid((ny + 255) / 256, nx);
    standard_kernel<Eq><<<grid, 256, 0, st>>>(cur, prev, out, frame, nx, ny, nv, gts, p);
}

struct SweptSet {
    SweptLaunch P, Y, G, O;
    bool fast = false;
};

template <int BX, bool GAP, class T = double, int VAR = 0, int MINROWS = 2>
void launch_fast(const SweptArgs& a, int grid, size_t smem, cudaStream_t st)
{
    auto k = heat_stream_fast<BX, GAP, T, VAR, MINROWS>;
    allow_big_smem(k);
    const int units = a.nb * a.nseg;
    // the per-cell courant variants add their operand ring to each warp's share
    if (VAR) smem = heat_fast_smem_v<BX, VAR>(a.Hmax);
    k<<<(units + kFastWarps - 1) / kFastWarps, 32 * kFastWarps, smem, st>>>(a);
}

// register-resident y-bridge seams of heat (seam_fast.cuh): one warp per
// column edge, the staged y-faces in shared memory
template <int BX>
void launch_yseam(const SweptArgs& a, int grid, size_t, cudaStream_t st)
{
    auto k = heat_yseam_fast<BX>;
    allow_big_smem(k);
    const int units = a.nb * a.nseg;
    k<<<(units + kSeamWarps - 1) / kSeamWarps, 32 * kSeamWarps, yseam_smem<BX>(a.Hmax), st>>>(a);
}

// register-resident octahedron seams of heat (seam_fast.cuh)
template <int BX>
void launch_oseam(const SweptArgs& a, int grid, size_t, cudaStream_t st)
{
    auto k = heat_oseam_fast<BX>;
    allow_big_smem(k);
    const int units = a.nb * a.nseg;
    k<<<(units + kSeamWarps - 1) / kSeamWarps, 32 * kSeamWarps, yseam_smem<BX>(a.Hmax), st>>>(a);
}

template <class Eq, int ITS, int W>
SweptSet make_set()
{
    return SweptSet{launch_stream<Eq, ITS, W, false>, launch_seam<Eq, ITS, false>,
                    launch_stream<Eq, ITS, W, true>, launch_seam<Eq, ITS, true>};
}

// (equation, ops, its, chunk) -> kernels; nullptr members = not built.
// Euler's stream tiles with the per-cell step (see EulerCell): an internal
// equation id for kernel selection only
constexpr int PS_EQ_EULER_CELL = 100;

bool pick_swept(int eq, int ops, int its, int chunk, SweptSet* out)
{
#define PS_SET(EQ, OP, IT, W, T) \
    if (eq == EQ && ops == OP && its == IT && chunk == W) { *out = make_set<T, IT, W>(); return true; }
    PS_SET(PS_EQ_HEAT, 1, 1, 32, Heat)
    PS_SET(PS_EQ_HEAT, 1, 2, 32, Heat)
    PS_SET(PS_EQ_HEAT, 1, 1, 64, Heat)
    PS_SET(PS_EQ_HEAT, 1, 2, 64, Heat)
    PS_SET(PS_EQ_EULER, 2, 2, 32, Euler)
    PS_SET(PS_EQ_EULER, 2, 2, 64, Euler)
    PS_SET(PS_EQ_EULER_CELL, 2, 2, 32, EulerCell)
    PS_SET(PS_EQ_EULER_CELL, 2, 2, 64, EulerCell)
    PS_SET(PS_EQ_HALF, 1, 1, 32, Half)
    PS_SET(PS_EQ_HALF, 1, 2, 32, Half)
    PS_SET(PS_EQ_EXAMPLE, 1, 1, 32, ExampleT<1>)
    PS_SET(PS_EQ_EXAMPLE, 1, 2, 32, ExampleT<1>)
    PS_SET(PS_EQ_EXAMPLE, 2, 1, 32, ExampleT<2>)
    PS_SET(PS_EQ_EXAMPLE, 2, 2, 32, ExampleT<2>)
    PS_SET(PS_EQ_CHECKER, 1, 1, 32, CheckerT<1>)
    PS_SET(PS_EQ_CHECKER, 1, 2, 32, CheckerT<1>)
    PS_SET(PS_EQ_CHECKER, 2, 1, 32, CheckerT<2>)
    PS_SET(PS_EQ_CHECKER, 2, 2, 32, CheckerT<2>)
    PS_SET(PS_EQ_HEATVAR, 1, 1, 32, HeatVar)
    PS_SET(PS_EQ_HEATVAR, 1, 1, 64, HeatVar)
    PS_SET(PS_EQ_HEATVAR_ADJ, 1, 1, 32, HeatVarAdj)
    PS_SET(PS_EQ_HEATVAR_ADJ, 1, 1, 64, HeatVarAdj)
    PS_SET(PS_EQ_HEATVAR_ADJMU, 1, 1, 32, HeatVarAdjMu)
    PS_SET(PS_EQ_HEATVAR_ADJMU, 1, 1, 64, HeatVarAdjMu)
#undef PS_SET
    return false;
}

StdLaunch pick_standard(int eq, int ops)
{
    switch (eq) {
    case PS_EQ_HEAT: return launch_standard<Heat>;
    case PS_EQ_EULER: return launch_standard<Euler>;
    case PS_EQ_HALF: return launch_standard<Half>;
    case PS_EQ_EXAMPLE: return ops == 2 ? launch_standard<ExampleT<2>> : launch_standard<ExampleT<1>>;
    case PS_EQ_CHECKER: return ops == 2 ? launch_standard<CheckerT<2>> : launch_standard<CheckerT<1>>;
    case PS_EQ_HEATVAR: return launch_standard<HeatVar>;
    case PS_EQ_HEATVAR_ADJ: return launch_standard<HeatVarAdj>;
    case PS_EQ_HEATVAR_ADJMU: return launch_standard<HeatVarAdjMu>;
    default: return nullptr;
    }
}

int check_launch(ps_solver* s)
{
    if (!s->launch_err.empty()) {
        const std::string m = s->launch_err;
        s->launch_err.clear();
        return fail(s, PS_ERR_CUDA, "kernel launch: %s", m.c_str());
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(s, PS_ERR_CUDA, "kernel launch: %s", cudaGetErrorString(e));
    s->launches++;
    return PS_OK;
}

cudaEvent_t take_event(ps_solver* s)
{
    if (!s->event_pool.empty()) {
        cudaEvent_t e = s->event_pool.back();
        s->event_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

// Kernel kinds for ps_profile_read: 0 prism stream, 1 Y-bridge seam, 2 gap
// stream, 3 octahedron seam, 4 standard step.
template <class F>
int timed_launch(ps_solver* s, int kind, double cells, F&& launch, cudaStream_t st = nullptr)
{
    cudaEvent_t a = nullptr, b = nullptr;
    if (!st) st = s->stream;
    if (s->profile) {
        a = take_event(s);
        b = take_event(s);
        cudaEventRecord(a, st);
    }
    launch();
    int rc = check_launch(s);
    if (s->profile) {
        cudaEventRecord(b, st);
        s->pending.push_back({kind, {a, b}});
        s->prof_cells[kind] += cells;
    }
    return rc;
}

int drain_profile(ps_solver* s)
{
    for (auto& p : s->pending) {
        float ms = 0.f;
        cudaError_t e = cudaEventElapsedTime(&ms, p.second.first, p.second.second);
        if (e != cudaSuccess) return fail(s, PS_ERR_CUDA, "event timing: %s", cudaGetErrorString(e));
        s->prof_ms[p.first] += ms;
        s->prof_n[p.first] += 1;
        s->event_pool.push_back(p.second.first);
        s->event_pool.push_back(p.second.second);
    }
    s->pending.clear();
    return PS_OK;
}

int ensure_swept_buffers(ps_solver* s)
{
    const int O2 = 2 * s->ops;
    const int nb = s->nx / s->bs;
    const int HF = std::max(s->H - 1, 0);
    const size_t xn = (size_t)nb * HF * 2 * s->nv * O2 * s->ny;
    // two y-face buffers: prism -> y-bridge, gap -> octahedron (the y-bridge
    // and the gap stream run at the same time)
    const size_t yn = 2 * (size_t)nb * s->nseg * 2 * HF * s->nv * s->bs * O2;
    if (xn > s->xface_n) {
        if (s->xface) cudaFree(s->xface);
        s->xface = nullptr;
        s->xface_n = 0;
        if (xn) PS_CUDA(s, cudaMalloc(&s->xface, nbytes(s, xn)));
        s->xface_n = xn;
    }
    if (yn > s->yface_n) {
        if (s->yface) cudaFree(s->yface);
        s->yface = nullptr;
        s->yface_n = 0;
        if (yn) PS_CUDA(s, cudaMalloc(&s->yface, nbytes(s, yn)));
        s->yface_n = yn;
    }
    return PS_OK;
}

// Levels per half-cycle until configured: MPSS, except heat with forward
// Euler at bs 32, whose register streams run fastest at 12 of the 15
// possible levels (measured on B200 at 4096² and 8192²: 3.8% and 6.9% over
// 15; the prism's last levels hold 2-6 rows and are pure latency).  Results
// do not depend on the choice.
int default_levels(int eq, int its, int bs, int mpss)
{
    // heat with forward Euler and the per-cell-courant variants share the
    // register streams, measured fastest at 12 levels for blocksize 32
    if ((eq == PS_EQ_HEAT || eq == PS_EQ_HEATVAR || eq == PS_EQ_HEATVAR_ADJMU) && its == 1 && bs == 32)
        return std::min(mpss, 12);
    return mpss;
}

// tile slots of the stream and seam kernels: a ring of its+1 for the built-in
// equations, levels -1 .. Hmax for a step hook (slot_count in swept.cuh)
int tile_slots(const ps_solver* s) { return s->hook ? s->H + 2 : s->its + 1; }

size_t stream_tile_smem(const ps_solver* s)
{
    const int O2 = 2 * s->ops, RS = s->chunk + O2;
    return s->esize * ((size_t)tile_slots(s) * s->nv * s->bs * RS +
                       (size_t)(s->H + 1) * s->nv * s->bs * O2);
}

// Euler streams share faces between cells when tile and scratch still leave
// room for two CTAs per SM (measured: with one CTA per SM the per-cell step
// on a wider chunk is faster; Euler stream levels are latency-bound)
constexpr size_t kFaceSmemCap = 113 * 1024;
bool euler_faces_fit(const ps_solver* s)
{
    return s->eq == PS_EQ_EULER &&
           stream_tile_smem(s) + sizeof(double) * euler_level_scratch(s->bs, s->chunk) <=
               kFaceSmemCap;
}

size_t stream_smem(const ps_solver* s)
{
    return stream_tile_smem(s) +
           (euler_faces_fit(s) ? sizeof(double) * euler_level_scratch(s->bs, s->chunk) : 0);
}

bool solver_seam_direct(const ps_solver* s)
{
    return seam_direct(s->bs, s->ops, s->nv, s->its, s->H, s->esize, tile_slots(s));
}

size_t seam_smem(const ps_solver* s)
{
    const int ns = tile_slots(s);
    if (solver_seam_direct(s))
        return s->esize * (size_t)ns * s->nv * s->bs * (2 * s->ops * (s->H + 1));
    return s->esize * std::max(seam_smem_elems(false, s->bs, s->ops, s->nv, s->its, s->H, ns),
                               seam_smem_elems(true, s->bs, s->ops, s->nv, s->its, s->H, ns));
}

// ------------------------------------------------------------ step hooks ----
// Driver-API launch of a hook kernel; a failure is kept for check_launch.
void hook_launch(ps_solver* s, CUfunction f, int gx, int gy, int nt, size_t smem,
                 cudaStream_t st, void** args)
{
    CUresult r = drv().launchKernel(f, gx, gy, 1, nt, 1, 1, (unsigned)smem, (CUstream)st, args,
                                    nullptr);
    if (r != CUDA_SUCCESS) s->launch_err = cu_error(r);
}

SweptSet hook_set(ps_solver* s)
{
    const int w = s->chunk == 64 ? 1 : 0;
    HookModule* h = s->hook;
    auto mk = [s](CUfunction f, int nt) {
        return [s, f, nt](const SweptArgs& a, int grid, size_t smem, cudaStream_t st) {
            SweptArgs copy = a;
            void* args[] = {&copy};
            hook_launch(s, f, grid, 1, nt, smem, st, args);
        };
    };
    return SweptSet{mk(h->prism[w], 256), mk(h->ybridge, 128), mk(h->gap[w], 256),
                    mk(h->octahedron, 128)};
}

// The framework constants of one kernel kind's tile (pysweep/core/pysweep.cu:
// 12-20, set by io.copyConstants, io.py:169-184): a tile of `rows` x `cols`
// cells per variable, levels `times` elements apart.
int hook_frame(ps_solver* s, int ns, int rows, int cols, int times)
{
    HookModule* h = s->hook;
    const int vals[FW_COUNT] = {rows * cols, times, s->mpss, 2 * s->mpss, s->nv,
                                s->ops,      s->its, rows,   cols};
    for (int f = 0; f < FW_COUNT; ++f) {
        CUresult r = hook_set_fw(h, ns, f, vals[f], (CUstream)s->stream);
        if (r != CUDA_SUCCESS)
            return fail(s, PS_ERR_CUDA, "hook constant %s: %s", kHookFw[f], cu_error(r).c_str());
    }
    return PS_OK;
}

int run_swept(ps_solver* s, int64_t nlevels, int gts0, double* frames, int64_t frame_cap,
              int frame_every)
{
    SweptSet K;
    const int keq = (s->eq == PS_EQ_EULER && !euler_faces_fit(s)) ? PS_EQ_EULER_CELL : s->eq;
    if (s->hook) {
        K = hook_set(s);
    } else if (!pick_swept(keq, s->ops, s->its, s->chunk, &K)) {
        return fail(s, PS_ERR_UNSUPPORTED, "no swept kernels for equation %d ops %d its %d chunk %d",
                    s->eq, s->ops, s->its, s->chunk);
    }
    const int O2 = 2 * s->ops;
    // register-resident streams for heat with forward Euler (the generic
    // seam kernels are shared)
    const bool fwd_euler = make_params(s).i[0] != 0;
    if (s->dtype == PS_DTYPE_F32) {
        // float32 fields: the register streams and the seams in float storage
        if (!(s->eq == PS_EQ_HEAT && s->its == 1 && fwd_euler && (s->bs == 16 || s->bs == 32) &&
              s->ny % 32 == 0))
            return fail(s, PS_ERR_UNSUPPORTED,
                        "float32 fields: heat, forward Euler, blocksize 16 or 32, ny a multiple of 32");
        K.fast = true;
        K.Y = launch_seam<HeatF32, 1, false, float>;
        K.O = launch_seam<HeatF32, 1, true, float>;
        K.P = s->bs == 16 ? launch_fast<16, false, float> : launch_fast<32, false, float>;
        K.G = s->bs == 16 ? launch_fast<16, true, float> : launch_fast<32, true, float>;
    } else if (!s->hook && s->eq == PS_EQ_HEAT && s->its == 1 && fwd_euler && s->threads != 256 &&
               (s->bs == 16 || s->bs == 32) && s->ny % 32 == 0) {
        K.fast = true;
        if (s->bs == 16) {
            K.P = launch_fast<16, false>;
            K.G = launch_fast<16, true>;
            K.Y = launch_yseam<16>;
            K.O = launch_oseam<16>;
        } else {
            // at most 14 levels per half-cycle: every prism level keeps 4 rows
            // or more, so its first 4 rows need no end test (8192², 1200
            // levels: 0.577 -> 0.570 ms per launch; 8 rows spilled)
            K.P = s->H <= 14 ? launch_fast<32, false, double, 0, 4> : launch_fast<32, false>;
            K.G = launch_fast<32, true>;
            K.Y = launch_yseam<32>;
            K.O = launch_oseam<32>;
        }
    } else if ((s->eq == PS_EQ_HEATVAR || s->eq == PS_EQ_HEATVAR_ADJMU) && s->threads != 256 &&
               (s->bs == 16 || s->bs == 32) && s->ny % 32 == 0) {
        // per-cell courant numbers in the register streams (the seams: the
        // generic kernels with the same equation's step_at)
        K.fast = true;
        if (s->eq == PS_EQ_HEATVAR) {
            K.P = s->bs == 16 ? launch_fast<16, false, double, 1> : launch_fast<32, false, double, 1>;
            K.G = s->bs == 16 ? launch_fast<16, true, double, 1> : launch_fast<32, true, double, 1>;
        } else {
            K.P = s->bs == 16 ? launch_fast<16, false, double, 2> : launch_fast<32, false, double, 2>;
            K.G = s->bs == 16 ? launch_fast<16, true, double, 2> : launch_fast<32, true, double, 2>;
        }
    }
    if (s->H < 1 || s->H > s->mpss) return fail(s, PS_ERR_INVALID, "levels per half-cycle %d not in [1, %d]", s->H, s->mpss);
    if (s->chunk < O2 * (s->H + 1))
        return fail(s, PS_ERR_INVALID, "chunk %d narrower than 2*ops*(h+1) = %d", s->chunk, O2 * (s->H + 1));
    if (K.fast) {
        if (s->nseg < 1 || s->nseg > s->ny / 32)
            return fail(s, PS_ERR_INVALID, "nseg %d not in [1, ny/32 = %d]", s->nseg, s->ny / 32);
    } else if (s->nseg < 1 || s->ny % s->nseg) {
        return fail(s, PS_ERR_INVALID, "ny %d not divisible into %d segments", s->ny, s->nseg);
    }
    // the first chunk of a segment shrinks by 2*ops per level on its left edge
    if (!K.fast && std::min(s->chunk, s->ny / s->nseg) < O2 * (s->H + 1))
        return fail(s, PS_ERR_INVALID, "segment width %d narrower than 2*ops*(h+1) = %d",
                    s->ny / s->nseg, O2 * (s->H + 1));
    if (s->nseg_auto) {
        if (K.fast) {
            // one warp per (band, segment); as many as the CTAs of 4 warps
            // that fit on the SMs at once (fast_ctas_per_sm)
            int sms = 148;
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
            const bool var = s->eq == PS_EQ_HEATVAR || s->eq == PS_EQ_HEATVAR_ADJMU;
            const int slots = sms * fast_ctas_per_sm(s->bs, var ? 1 : 0) * kFastWarps;
            const int nb = s->nx / s->bs;
            s->nseg = std::max(1, std::min(s->ny / kFastChunk, slots / nb));
            s->nseg = std::max(1, std::min(s->nseg, s->ny / 32));
        } else {
            // one CTA per (band, segment): the most segments that divide ny
            // and keep four chunks (and 2*ops*(h+1) columns) each.  Shorter
            // segments make the seams as costly as the streams; longer ones
            // leave few, long CTAs and a ragged last wave.  Measured on Euler
            // (G cell-stages/s): 1024², bs 32: 16 segments 3.00, 8: 3.31,
            // 4: 3.32; 4096², bs 16: 2: 5.65, 16: 6.26, 32: 5.93, 64: 5.39.
            // Step hooks keep eight chunks where that still gives every SM a
            // CTA: their seams are the generic ones, with a slot per level
            // (heat as a hook at 4096², Gcell-updates/s: bs 16, 32 segments
            // 105.5, 16: 113.3; bs 32 at h 6: 128.5 and 135.6).
            int sms = 148;
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
            int minw = std::max(4 * s->chunk, O2 * (s->H + 1));
            if (s->hook && (s->nx / s->bs) * (s->ny / (8 * s->chunk)) >= sms)
                minw = std::max(minw, 8 * s->chunk);
            s->nseg = 1;
            for (int q = 2; s->ny / q >= minw; ++q)
                if (s->ny % q == 0) s->nseg = q;
        }
    }
    const size_t smem = std::max(stream_smem(s), seam_smem(s));
    if (smem > 227 * 1024)
        return fail(s, PS_ERR_UNSUPPORTED, "tile needs %zu bytes of shared memory", smem);
    int rc = ensure_swept_buffers(s);
    if (rc) return rc;
    if (!s->side) {
        int lo = 0, hi = 0;
        PS_CUDA(s, cudaDeviceGetStreamPriorityRange(&lo, &hi));
        PS_CUDA(s, cudaStreamCreateWithPriority(&s->side, cudaStreamNonBlocking, hi));
        PS_CUDA(s, cudaEventCreateWithFlags(&s->ev_fork, cudaEventDisableTiming));
        PS_CUDA(s, cudaEventCreateWithFlags(&s->ev_join, cudaEventDisableTiming));
    }
    SweptArgs a;
    memset(&a, 0, sizeof a);
    a.frames = frames;
    a.frame_cap = frames ? frame_cap : 0;
    a.frame_every = frame_every > 0 ? frame_every : 1;
    a.nx = s->nx;
    a.ny = s->ny;
    a.nv = s->nv;
    a.bx = s->bs;
    a.hx = s->bs / 2;
    a.Hmax = s->H;
    a.nb = s->nx / s->bs;
    a.nseg = s->nseg;
    a.wy = s->ny / s->nseg;
    // the last chunk may be partial (generic streams); the register streams
    // use whole 64-column chunks
    a.nchunks = K.fast ? a.wy / kFastChunk : (a.wy + s->chunk - 1) / s->chunk;
    a.seg_unit = K.fast ? 32 : a.wy;
    a.seg_units = K.fast ? s->ny / 32 : s->nseg;
    a.its = s->its;
    a.gts_base = gts0 - 1;
    a.xface = s->xface;
    a.yface = s->yface;
    a.p = make_params(s);
    a.seam_direct = solver_seam_direct(s) ? 1 : 0;
    const int units = a.nb * a.nseg;
    if (s->hook) {
        // the hook's tiles: stream slots of bs rows x (chunk + 2 OPS) columns
        // whose levels sit one slot + OPS apart (the chunk's parallelogram),
        // seam slots of bs rows x 2 OPS (Hmax + 1) columns, one slot apart
        const int rs = s->chunk + O2, tw = 2 * s->ops * (s->H + 1);
        if ((rc = hook_frame(s, HOOK_STREAM, s->bs, rs, s->nv * s->bs * rs + s->ops)) ||
            (rc = hook_frame(s, HOOK_SEAM, s->bs, tw, s->nv * s->bs * tw)))
            return rc;
    }
    const size_t fe = field_elems(s);
    int off = 0;
    int64_t done = 0;
    while (done < nlevels) {
        const int H = (int)std::min<int64_t>(s->H, nlevels - done);
        a.H = H;
        a.L0 = done;
        a.off = off;
        a.bin = s->base[s->cur];
        a.bout = s->base[1 - s->cur];
        if (H < s->its) {
            // the newest its-H base levels carry over unchanged
            for (int q = 0; q < s->its - H; ++q)
                PS_CUDA(s, cudaMemcpyAsync(at(s, s->base[1 - s->cur], (size_t)q * fe),
                                           at(s, s->base[s->cur], (size_t)(q + H) * fe),
                                           nbytes(s, fe), cudaMemcpyDeviceToDevice, s->stream));
        }
        // algorithmic cell updates of each kernel in this half-cycle
        double cP = 0, cY = 0, cG = 0, cO = 0;
        for (int m = 1; m <= H; ++m) {
            const double rp = s->bs - 2.0 * s->ops * m, rg = 2.0 * s->ops * m;
            const double cm = 2.0 * s->ops * m * s->nseg;  // seam columns of a band
            const double cs = (double)s->ny - cm;           // stream columns of a band
            cP += rp * cs;
            cY += rp * cm;
            cG += rg * cs;
            cO += rg * cm;
        }
        const double u = (double)a.nb;
        const size_t psm = K.fast ? (s->bs == 16 ? heat_fast_smem<16>(s->H) : heat_fast_smem<32>(s->H))
                                  : stream_smem(s);
        // P, then Y on `stream` beside G on the side stream (G reads nothing
        // that Y writes: its valid cells depend on the prisms' faces only,
        // and adjacent bands share their segment boundaries, so G's
        // trapezoids avoid both bands' y-bridge diamonds; it writes its
        // y-faces into the second buffer), then O
        SweptArgs ag = a;
        ag.yface = at(s, s->yface, s->yface_n / 2);
        if ((rc = timed_launch(s, 0, cP * u, [&] { K.P(a, units, psm, s->stream); }))) return rc;
        PS_CUDA(s, cudaEventRecord(s->ev_fork, s->stream));
        PS_CUDA(s, cudaStreamWaitEvent(s->side, s->ev_fork, 0));
        if ((rc = timed_launch(s, 2, cG * u, [&] { K.G(ag, units, psm, s->side); }, s->side))) return rc;
        PS_CUDA(s, cudaEventRecord(s->ev_join, s->side));
        if ((rc = timed_launch(s, 1, cY * u, [&] { K.Y(a, units, seam_smem(s), s->stream); }))) return rc;
        PS_CUDA(s, cudaStreamWaitEvent(s->stream, s->ev_join, 0));
        if ((rc = timed_launch(s, 3, cO * u, [&] { K.O(ag, units, seam_smem(s), s->stream); }))) return rc;
        s->cur = 1 - s->cur;
        off = ((off - a.hx) % s->nx + s->nx) % s->nx;
        done += H;
    }
    return PS_OK;
}

int run_standard(ps_solver* s, int64_t nlevels, int gts0, double* frames, int64_t frame_cap,
                 int frame_every)
{
    StdLaunch K = s->hook ? nullptr : pick_standard(s->eq, s->ops);
    if (!K && !s->hook) return fail(s, PS_ERR_UNSUPPORTED, "no standard kernel for equation %d", s->eq);
    const size_t fe = field_elems(s);
    for (int i = 0; i < 3; ++i)
        if (!s->ring[i]) PS_CUDA(s, cudaMalloc(&s->ring[i], nbytes(s, fe)));
    const int its = s->its;
    // ring[c] = current level, ring[p] = previous level
    int c = 0, p = 1, n = 2;
    double* b = s->base[s->cur];
    PS_CUDA(s, cudaMemcpyAsync(s->ring[c], at(s, b, (size_t)(its - 1) * fe), nbytes(s, fe),
                               cudaMemcpyDeviceToDevice, s->stream));
    PS_CUDA(s, cudaMemcpyAsync(s->ring[p], at(s, b, (size_t)(its >= 2 ? its - 2 : 0) * fe),
                               nbytes(s, fe), cudaMemcpyDeviceToDevice, s->stream));
    const EqParams prm = make_params(s);
    const int every = frame_every > 0 ? frame_every : 1;
    // streaming heat kernel (64-column strips); threads = 256 keeps the generic one
    const bool fast = s->eq == PS_EQ_HEAT && s->ny % 64 == 0 && s->threads != 256;
    const bool f32 = s->dtype == PS_DTYPE_F32;
    // Euler: faces shared between cells (threads = 256 keeps the per-cell kernel)
    const bool euler_faces = s->eq == PS_EQ_EULER && s->threads != 256;
    if (euler_faces) allow_big_smem(euler_standard_faces);
    if (f32 && !(fast && prm.i[0]))
        return fail(s, PS_ERR_UNSUPPORTED,
                    "float32 fields: heat with forward Euler and ny a multiple of 64 only");
    int rc;
    if (s->hook) {
        // the hook's standard tile: kHookStdTR x kHookStdTC cells and an
        // OPS-cell halo per variable, previous / current / next level one slot apart
        const int tr = kHookStdTR + 2 * s->ops, tc = kHookStdTC + 2 * s->ops;
        if ((rc = hook_frame(s, HOOK_STD, tr, tc, s->nv * tr * tc))) return rc;
    }
    for (int64_t L = 1; L <= nlevels; ++L) {
        double* fr = nullptr;
        if (frames && L % its == 0 && (L / its) % every == 0) {
            const int64_t slot = (L / its) / every - 1;
            if (slot < frame_cap) fr = at(s, frames, (size_t)slot * fe);
        }
        const int gts = gts0 + (int)(L - 1);
        if ((rc = timed_launch(s, 4, (double)s->nx * s->ny, [&] {
                 if (s->hook) {
                     const double* cur = s->ring[c];
                     const double* prv = s->ring[p];
                     double* nxt = s->ring[n];
                     int nx = s->nx, ny = s->ny, g = gts;
                     void* args[] = {&cur, &prv, &nxt, &fr, &nx, &ny, &g};
                     const size_t tr = kHookStdTR + 2 * s->ops, tc = kHookStdTC + 2 * s->ops;
                     hook_launch(s, s->hook->standard, (s->ny + kHookStdTC - 1) / kHookStdTC,
                                 (s->nx + kHookStdTR - 1) / kHookStdTR, kHookStdNT,
                                 3 * sizeof(double) * s->nv * tr * tc, s->stream, args);
                 } else if (fast) {
                     const dim3 grid((s->ny / 64 + 7) / 8, (s->nx + kStdRows - 1) / kStdRows);
                     if (f32)
                         heat_standard_fast<false, float><<<grid, 256, 0, s->stream>>>(
                             (const float*)s->ring[c], (const float*)s->ring[p], (float*)s->ring[n],
                             (float*)fr, s->nx, s->ny, gts, prm.d[0]);
                     else if (prm.i[0])
                         heat_standard_fast<false><<<grid, 256, 0, s->stream>>>(
                             s->ring[c], s->ring[p], s->ring[n], fr, s->nx, s->ny, gts, prm.d[0]);
                     else
                         heat_standard_fast<true><<<grid, 256, 0, s->stream>>>(
                             s->ring[c], s->ring[p], s->ring[n], fr, s->nx, s->ny, gts, prm.d[0]);
                 } else if (euler_faces) {
                     const dim3 grid((s->ny + kEuTC - 1) / kEuTC, (s->nx + kEuTR - 1) / kEuTR);
                     euler_standard_faces<<<grid, 256, kEuStdSmem, s->stream>>>(
                         s->ring[c], s->ring[p], s->ring[n], fr, s->nx, s->ny, gts, prm);
                 } else {
                     K(s->ring[c], s->ring[p], s->ring[n], fr, s->nx, s->ny, s->nv, gts, prm,
                       s->stream);
                 }
             })))
            return rc;
        const int t = p;
        p = c;
        c = n;
        n = t;
    }
    // newest levels back into the base
    PS_CUDA(s, cudaMemcpyAsync(at(s, b, (size_t)(its - 1) * fe), s->ring[c], nbytes(s, fe),
                               cudaMemcpyDeviceToDevice, s->stream));
    if (its >= 2)
        PS_CUDA(s, cudaMemcpyAsync(at(s, b, (size_t)(its - 2) * fe), s->ring[p], nbytes(s, fe),
                                   cudaMemcpyDeviceToDevice, s->stream));
    return PS_OK;
}

struct GlobalSpec {
    const char* name;
    int eqmask;  // bit per equation
};

const GlobalSpec kGlobals[] = {
    {"DT", 0x1f},    {"DX", 0x1f},      {"DY", 0x1f},   {"ALPHA", 1 << PS_EQ_HEAT},
    {"SCHEME", (1 << PS_EQ_HEAT) | (1 << PS_EQ_EXAMPLE) | (1 << PS_EQ_CHECKER)},
    {"GAMMA", 1 << PS_EQ_EULER}, {"GAM_M1", 1 << PS_EQ_EULER}, {"DTDX", 1 << PS_EQ_EULER},
    {"DTDY", 1 << PS_EQ_EULER}, {"LEN", (1 << PS_EQ_HEATVAR) | (1 << PS_EQ_HEATVAR_ADJ) | (1 << PS_EQ_HEATVAR_ADJMU)},
};

const GlobalSpec* find_global(const ps_solver* s, const char* name)
{
    for (const auto& g : kGlobals)
        if (!strcmp(g.name, name) && (g.eqmask >> s->eq & 1)) return &g;
    return nullptr;
}

double decode_value(const void* value, size_t nbytes)
{
    switch (nbytes) {
    case 8: {
        double d;
        memcpy(&d, value, 8);
        return d;
    }
    case 4: {
        int32_t i;
        memcpy(&i, value, 4);
        return (double)i;
    }
    case 2: {
        int16_t i;
        memcpy(&i, value, 2);
        return (double)i;
    }
    case 1: return (double)*(const uint8_t*)value;
    default: return 0.0;
    }
}

int solver_open(ps_solver* s);

// Kind of a hook constant, from its declaration in the hook's source:
// 'f' floating point, 'b' bool, 'i' any other (integer) type.
char hook_const_kind(const std::string& src, const std::string& name)
{
    size_t pos = 0;
    while ((pos = src.find("__constant__", pos)) != std::string::npos) {
        const size_t end = src.find(';', pos);
        if (end == std::string::npos) break;
        const std::string decl = src.substr(pos, end - pos);
        pos = end;
        // the name as a whole word of the declaration
        size_t k = 0;
        bool found = false;
        while ((k = decl.find(name, k)) != std::string::npos) {
            const bool l = k == 0 || !(isalnum((unsigned char)decl[k - 1]) || decl[k - 1] == '_');
            const size_t e = k + name.size();
            const bool r = e >= decl.size() || !(isalnum((unsigned char)decl[e]) || decl[e] == '_');
            if (l && r) {
                found = true;
                break;
            }
            k = e;
        }
        if (!found) continue;
        if (decl.find("double") != std::string::npos || decl.find("float") != std::string::npos)
            return 'f';
        if (decl.find("bool") != std::string::npos) return 'b';
        return 'i';
    }
    return 'f';
}

// The value in the representation of a hook constant of `size` bytes and
// `kind` (the caller's bytes as they are when the sizes agree, else converted
// through double).
bool hook_encode(const void* value, size_t nbytes, size_t size, char kind, unsigned char* buf)
{
    if (nbytes == size) {
        memcpy(buf, value, size);
        return true;
    }
    const double d = decode_value(value, nbytes);
    if (kind == 'f' && size == 8) {
        memcpy(buf, &d, 8);
    } else if (kind == 'f' && size == 4) {
        const float f = (float)d;
        memcpy(buf, &f, 4);
    } else if (size == 8) {
        const int64_t i = (int64_t)d;
        memcpy(buf, &i, 8);
    } else if (size == 4) {
        const int32_t i = (int32_t)d;
        memcpy(buf, &i, 4);
    } else if (size == 2) {
        const int16_t i = (int16_t)d;
        memcpy(buf, &i, 2);
    } else if (size == 1) {
        buf[0] = kind == 'b' ? (d != 0.0) : (unsigned char)(int)d;
    } else {
        return false;
    }
    return true;
}

}  // namespace

extern "C" {

const char* ps_version(void) { return kVersion; }

const char* ps_last_error(const ps_solver* s)
{
    return s ? s->err.c_str() : g_create_error.c_str();
}

int64_t ps_kernel_launches(const ps_solver* s) { return s ? s->launches : 0; }

int ps_create(ps_solver** out, int device, int equation, int nv, int nx, int ny, int ops, int its,
              int blocksize)
{
    return ps_create_typed(out, device, equation, nv, nx, ny, ops, its, blocksize, PS_DTYPE_F64);
}

int ps_create_typed(ps_solver** out, int device, int equation, int nv, int nx, int ny, int ops,
                    int its, int blocksize, int dtype)
{
    if (!out) return PS_ERR_INVALID;
    *out = nullptr;
    if (equation < PS_EQ_HEAT || equation > PS_EQ_HEATVAR_ADJMU || equation == PS_EQ_HOOK)
        return PS_ERR_INVALID;
    if (dtype != PS_DTYPE_F64 && dtype != PS_DTYPE_F32) return PS_ERR_INVALID;
    ps_solver* s = new ps_solver();
    s->dtype = dtype;
    s->esize = dtype == PS_DTYPE_F32 ? sizeof(float) : sizeof(double);
    s->device = device;
    s->eq = equation;
    s->nv = nv;
    s->nx = nx;
    s->ny = ny;
    s->ops = eq_ops(equation, ops);
    s->its = its;
    s->bs = blocksize;
    int rc = PS_OK;
    if (equation == PS_EQ_HEAT || equation == PS_EQ_HALF) {
        if (nv != 1) rc = fail(s, PS_ERR_INVALID, "heat/half have one variable, got nv=%d", nv);
    }
    if (((equation == PS_EQ_HEATVAR || equation == PS_EQ_HEATVAR_ADJMU) && nv != 1) ||
        (equation == PS_EQ_HEATVAR_ADJ && nv != 2) ||
        ((equation == PS_EQ_HEATVAR || equation == PS_EQ_HEATVAR_ADJ || equation == PS_EQ_HEATVAR_ADJMU) &&
         its != 1))
        rc = fail(s, PS_ERR_INVALID,
                  "heatvar and its mu-form adjoint have nv=1, the lambda-form adjoint nv=2; its=1 "
                  "(got nv=%d its=%d)", nv, its);
    if (equation == PS_EQ_EULER && (nv != 4 || its != 2))
        rc = fail(s, PS_ERR_INVALID, "euler needs nv=4 and its=2 (got nv=%d its=%d)", nv, its);
    if (ops != s->ops) rc = fail(s, PS_ERR_INVALID, "equation %d has ops=%d, got %d", equation, s->ops, ops);
    if (dtype == PS_DTYPE_F32 && (equation != PS_EQ_HEAT || its != 1))
        rc = fail(s, PS_ERR_UNSUPPORTED, "float32 fields: heat with forward Euler (its=1) only");
    if (nv < 1 || nv > 4 || its < 1 || its > 2 || ops < 1 || ops > 2)
        rc = fail(s, PS_ERR_UNSUPPORTED, "nv in 1..4, its in 1..2, ops in 1..2 supported");
    if (blocksize <= 0 || blocksize % (2 * s->ops))  // io.py:52
        rc = fail(s, PS_ERR_INVALID, "blocksize %d must be a multiple of 2*ops", blocksize);
    if (rc == PS_OK && (nx % blocksize || ny % blocksize))  // process.py:143
        rc = fail(s, PS_ERR_INVALID, "array %dx%d not divisible by blocksize %d", nx, ny, blocksize);
    if (rc == PS_OK && (size_t)3 * nv * nx * ny >= (size_t)1 << 31)
        rc = fail(s, PS_ERR_UNSUPPORTED, "field too large for 32-bit offsets");
    s->mpss = blocksize / (2 * s->ops) - 1;
    if (rc == PS_OK && s->mpss < 1)
        rc = fail(s, PS_ERR_INVALID, "blocksize %d gives no swept level (MPSS < 1)", blocksize);
    s->H = default_levels(s->eq, s->its, blocksize, s->mpss);
    s->chunk = (2 * s->ops * (s->H + 1) <= 32) ? 32 : 64;
    // Euler: 64-column chunks keep every thread of a stream CTA busy on each
    // level, where the tile fits in shared memory
    if (s->eq == PS_EQ_EULER && s->chunk == 32) {
        s->chunk = 64;
        if (stream_smem(s) > 227 * 1024) s->chunk = 32;
    }
    if (rc == PS_OK) rc = solver_open(s);
    if (rc != PS_OK) {
        g_create_error = s->err;  // readable through ps_last_error(NULL)
        ps_destroy(s);
        return rc;
    }
    *out = s;
    return PS_OK;
}

}  // extern "C"

namespace {

// The device half of solver creation: device, stream, base buffers.
int solver_open(ps_solver* s)
{
    const int device = s->device, nv = s->nv, nx = s->nx, ny = s->ny, its = s->its;
    int rc = PS_OK;
    s->nseg = 1;
    if (rc == PS_OK) {
        cudaError_t e = cudaSetDevice(device);
        if (e != cudaSuccess) rc = fail(s, PS_ERR_CUDA, "cudaSetDevice: %s", cudaGetErrorString(e));
    }
    if (rc == PS_OK) {
        cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) rc = fail(s, PS_ERR_CUDA, "cudaStreamCreate: %s", cudaGetErrorString(e));
        s->own_stream = true;
    }
    if (rc == PS_OK) {
        const size_t bytes = nbytes(s, (size_t)its * nv * nx * ny);
        for (int i = 0; i < 2 && rc == PS_OK; ++i) {
            cudaError_t e = cudaMalloc(&s->base[i], bytes);
            if (e != cudaSuccess) rc = fail(s, PS_ERR_NOMEM, "cudaMalloc base: %s", cudaGetErrorString(e));
        }
    }
    return rc;
}

}  // namespace

extern "C" {

int ps_hook_check(const char* source, const char* name, int nv, int ops, int its, char* log,
                  size_t loglen)
{
    if (log && loglen) log[0] = '\0';
    if (!source || nv < 1 || nv > 8 || ops < 1 || ops > 4 || its < 1 || its > 2)
        return PS_ERR_INVALID;
    std::vector<char> cubin;
    std::string lg;
    const int rc = hook_compile(hook_program(source, name ? name : "hook.cu", nv, ops, its), &cubin, &lg);
    if (log && loglen) {
        strncpy(log, lg.c_str(), loglen - 1);
        log[loglen - 1] = '\0';
    }
    return rc;
}

int ps_create_hook(ps_solver** out, int device, const char* source, const char* name, int nv,
                   int nx, int ny, int ops, int its, int blocksize)
{
    if (!out) return PS_ERR_INVALID;
    *out = nullptr;
    ps_solver* s = new ps_solver();
    s->device = device;
    s->eq = PS_EQ_HOOK;
    s->nv = nv;
    s->nx = nx;
    s->ny = ny;
    s->ops = ops;
    s->its = its;
    s->bs = blocksize;
    int rc = PS_OK;
    if (!source) rc = fail(s, PS_ERR_INVALID, "no hook source");
    else if (nv < 1 || nv > 8 || ops < 1 || ops > 4 || its < 1 || its > 2)
        rc = fail(s, PS_ERR_UNSUPPORTED, "step hooks: nv in 1..8, ops in 1..4, its in 1..2");
    else if (blocksize <= 0 || blocksize % (2 * ops))  // io.py:52
        rc = fail(s, PS_ERR_INVALID, "blocksize %d must be a multiple of 2*ops", blocksize);
    else if (nx <= 0 || ny <= 0 || nx % blocksize || ny % blocksize)  // process.py:143
        rc = fail(s, PS_ERR_INVALID, "array %dx%d not divisible by blocksize %d", nx, ny, blocksize);
    else if ((size_t)3 * nv * nx * ny >= (size_t)1 << 31)
        rc = fail(s, PS_ERR_UNSUPPORTED, "field too large for 32-bit offsets");
    s->mpss = blocksize > 0 && ops > 0 ? blocksize / (2 * ops) - 1 : 0;
    if (rc == PS_OK && s->mpss < 1)
        rc = fail(s, PS_ERR_INVALID, "blocksize %d gives no swept level (MPSS < 1)", blocksize);
    if (rc == PS_OK) {
        s->hook = new HookModule();
        s->hook->nv = nv;
        s->hook->ops = ops;
        s->hook->its = its;
        s->hook_src = source;
        // levels per half-cycle: the most (up to MPSS) whose stream tile,
        // one linear slot per level, leaves room for three CTAs per SM; where
        // none does, the most that fit at all.  (The heat plugin as a hook,
        // 4096², 600 steps, Gcell-updates/s: bs 32 at MPSS = 15, one CTA per
        // SM, 59; at 6, three CTAs, 136; bs 16 keeps MPSS = 7.)
        for (const size_t cap : {(size_t)227 * 1024 / 3, (size_t)227 * 1024}) {
            s->H = s->mpss;
            bool fits = false;
            for (;;) {
                s->chunk = (2 * ops * (s->H + 1) <= 32) ? 32 : 64;
                fits = 2 * ops * (s->H + 1) <= 64 && stream_smem(s) <= cap &&
                       seam_smem(s) <= 227 * 1024;
                if (fits || s->H == 1) break;
                --s->H;
            }
            if (fits) break;
        }
        std::vector<char> cubin;
        std::string log;
        rc = hook_compile(hook_program(source, name ? name : "hook.cu", nv, ops, its), &cubin, &log);
        if (rc) fail(s, PS_ERR_COMPILE, "step hook %s did not compile:\n%s", name ? name : "", log.c_str());
        if (rc == PS_OK) rc = solver_open(s);  // device, stream (the primary context), bases
        if (rc == PS_OK) {
            std::string err;
            if (hook_load(s->hook, cubin, &err)) rc = fail(s, PS_ERR_CUDA, "%s", err.c_str());
        }
    }
    if (rc != PS_OK) {
        g_create_error = s->err;
        ps_destroy(s);
        return rc;
    }
    *out = s;
    return PS_OK;
}

int ps_destroy(ps_solver* s)
{
    if (!s) return PS_OK;
    cudaSetDevice(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    for (auto& b : s->base)
        if (b) cudaFree(b);
    for (auto& r : s->ring)
        if (r) cudaFree(r);
    if (s->xface) cudaFree(s->xface);
    if (s->yface) cudaFree(s->yface);
    if (s->hook) {
        if (s->hook->mod) drv().moduleUnload(s->hook->mod);
        delete s->hook;
    }
    for (auto& p : s->pending) {
        cudaEventDestroy(p.second.first);
        cudaEventDestroy(p.second.second);
    }
    for (auto e : s->event_pool) cudaEventDestroy(e);
    if (s->side) {
        cudaStreamSynchronize(s->side);
        cudaStreamDestroy(s->side);
    }
    if (s->ev_fork) cudaEventDestroy(s->ev_fork);
    if (s->ev_join) cudaEventDestroy(s->ev_join);
    if (s->own_stream && s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return PS_OK;
}

int ps_set_global(ps_solver* s, const char* name, const void* value, size_t nbytes)
{
    if (!s || !name || !value) return PS_ERR_INVALID;
    if (nbytes != 1 && nbytes != 2 && nbytes != 4 && nbytes != 8)
        return fail(s, PS_ERR_INVALID, "constant %s: unsupported size %zu", name, nbytes);
    if (s->hook) {
        // the hook's own __constant__, in every kernel kind's copy, written in
        // stream order (kernels queued before keep the old value)
        PS_CUDA(s, cudaSetDevice(s->device));
        HookConst* c = hook_const(s->hook, name);
        if (!c) return fail(s, PS_ERR_INVALID, "the step hook declares no __constant__ %s", name);
        unsigned char buf[8];
        if (!hook_encode(value, nbytes, c->size, hook_const_kind(s->hook_src, name), buf))
            return fail(s, PS_ERR_UNSUPPORTED, "constant %s: %zu-byte type", name, c->size);
        for (int k = 0; k < 3; ++k) {
            CUresult r = drv().memcpyHtoDAsync(c->ptr[k], buf, c->size, (CUstream)s->stream);
            if (r != CUDA_SUCCESS)
                return fail(s, PS_ERR_CUDA, "constant %s: %s", name, cu_error(r).c_str());
        }
        s->globals[name] = decode_value(value, nbytes);
        return PS_OK;
    }
    if (!find_global(s, name)) return fail(s, PS_ERR_INVALID, "no constant named %s", name);
    s->globals[name] = decode_value(value, nbytes);
    return PS_OK;
}

int ps_get_global(ps_solver* s, const char* name, void** handle, size_t* size)
{
    if (!s || !name) return PS_ERR_INVALID;
    if (s->hook) {
        PS_CUDA(s, cudaSetDevice(s->device));
        HookConst* c = hook_const(s->hook, name);
        if (!c) return fail(s, PS_ERR_INVALID, "the step hook declares no __constant__ %s", name);
        if (handle) *handle = (void*)c;  // `name` first, like the built-ins' GlobalSpec
        if (size) *size = c->size;
        return PS_OK;
    }
    const GlobalSpec* g = find_global(s, name);
    if (!g) return fail(s, PS_ERR_INVALID, "no constant named %s", name);
    if (handle) *handle = (void*)g;
    if (size) *size = !strcmp(name, "SCHEME") ? 4 : 8;
    return PS_OK;
}

int ps_set_global_handle(ps_solver* s, void* handle, const void* value, size_t nbytes)
{
    if (!s || !handle) return PS_ERR_INVALID;
    return ps_set_global(s, ((const GlobalSpec*)handle)->name, value, nbytes);
}

int ps_get_global_value(ps_solver* s, const char* name, double* value)
{
    if (!s || !name || !value) return PS_ERR_INVALID;
    const int SX = s->nx, SY = s->ny;
    const int T = 2 * s->mpss + s->its;
    if (!strcmp(name, "NV")) *value = s->nv;
    else if (!strcmp(name, "SX")) *value = SX;
    else if (!strcmp(name, "SY")) *value = SY;
    else if (!strcmp(name, "VARS")) *value = (double)SX * SY;
    else if (!strcmp(name, "TIMES")) *value = (double)s->nv * SX * SY;
    else if (!strcmp(name, "MPSS")) *value = s->mpss;
    else if (!strcmp(name, "MOSS")) *value = 2 * s->mpss;
    else if (!strcmp(name, "OPS")) *value = s->ops;
    else if (!strcmp(name, "ITS")) *value = s->its;
    else if (!strcmp(name, "T")) *value = T;
    else {
        auto it = s->globals.find(name);
        if (it == s->globals.end()) return fail(s, PS_ERR_INVALID, "no constant named %s", name);
        *value = it->second;
    }
    return PS_OK;
}

int ps_configure(ps_solver* s, int h, int nseg, int chunk, int threads)
{
    if (!s) return PS_ERR_INVALID;
    if (h < 0 || nseg < 0 || chunk < 0 || threads < 0) return fail(s, PS_ERR_INVALID, "negative knob");
    if (h) {
        if (h > s->mpss) return fail(s, PS_ERR_INVALID, "h %d > MPSS %d", h, s->mpss);
        s->H = h;
    }
    if (nseg) {
        s->nseg = nseg;
        s->nseg_auto = false;
    }
    if (chunk) {
        if (chunk != 32 && chunk != 64) return fail(s, PS_ERR_INVALID, "chunk must be 32 or 64");
        s->chunk = chunk;
    }
    if (threads) {
        // 128: register-resident heat streams where they apply (default);
        // 256: always the generic shared-memory streams
        if (threads != 256 && threads != 128)
            return fail(s, PS_ERR_UNSUPPORTED, "threads must be 128 or 256");
        s->threads = threads;
    }
    return PS_OK;
}

int ps_get_tiling(ps_solver* s, int* h, int* nseg, int* chunk, int* mpss)
{
    if (!s) return PS_ERR_INVALID;
    if (h) *h = s->H;
    if (nseg) *nseg = s->nseg;
    if (chunk) *chunk = s->chunk;
    if (mpss) *mpss = s->mpss;
    return PS_OK;
}

int ps_set_state(ps_solver* s, const double* src, int levels, int src_on_device)
{
    if (!s || !src) return PS_ERR_INVALID;
    if (levels != 1 && levels != s->its)
        return fail(s, PS_ERR_INVALID, "levels must be 1 or its=%d", s->its);
    PS_CUDA(s, cudaSetDevice(s->device));
    const size_t fe = field_elems(s);
    const cudaMemcpyKind kind = src_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    for (int q = 0; q < s->its; ++q) {
        const double* from = at(s, const_cast<double*>(src), (size_t)(levels == 1 ? 0 : q) * fe);
        PS_CUDA(s, cudaMemcpyAsync(at(s, s->base[s->cur], (size_t)q * fe), from, nbytes(s, fe),
                                   kind, s->stream));
    }
    if (!src_on_device) PS_CUDA(s, cudaStreamSynchronize(s->stream));
    s->have_state = true;
    return PS_OK;
}

int ps_set_field(ps_solver* s, int index, double* d_field)
{
    if (!s) return PS_ERR_INVALID;
    if (s->eq != PS_EQ_HEATVAR && s->eq != PS_EQ_HEATVAR_ADJ && s->eq != PS_EQ_HEATVAR_ADJMU)
        return fail(s, PS_ERR_INVALID, "equation %d reads no grid fields", s->eq);
    if (index < 0 || index > 2) return fail(s, PS_ERR_INVALID, "field index %d not 0, 1 or 2", index);
    s->field[index] = d_field;
    return PS_OK;
}

int ps_run(ps_solver* s, int mode, int64_t nlevels, int gts0, double* frames, int64_t frame_cap,
           int frame_every, int frames_on_device)
{
    if (!s) return PS_ERR_INVALID;
    if (!s->have_state) return fail(s, PS_ERR_STATE, "ps_run before ps_set_state");
    if (nlevels < 0) return fail(s, PS_ERR_INVALID, "negative level count");
    if (frame_every < 0) return fail(s, PS_ERR_INVALID, "negative frame_every");
    const bool hv = s->eq == PS_EQ_HEATVAR || s->eq == PS_EQ_HEATVAR_ADJ || s->eq == PS_EQ_HEATVAR_ADJMU;
    if (hv && !s->field[0]) return fail(s, PS_ERR_STATE, "heatvar: no courant field (ps_set_field 0)");
    if ((s->eq == PS_EQ_HEATVAR_ADJ || s->eq == PS_EQ_HEATVAR_ADJMU) && !s->field[1])
        return fail(s, PS_ERR_STATE, "heatvar adjoint: no recomputed Laplacians (ps_set_field 1)");
    if (s->eq == PS_EQ_HEATVAR_ADJMU && !s->field[2])
        return fail(s, PS_ERR_STATE, "heatvar adjoint (mu): no sum field (ps_set_field 2)");
    if (hv && s->field[1] && nlevels > 0) {
        // field 1 holds LEN levels: the run's levels gts0 .. gts0+nlevels-1 must index them
        auto it = s->globals.find("LEN");
        const int64_t len = it == s->globals.end() ? 0 : (int64_t)it->second;
        if (gts0 < 1 || gts0 - 1 + nlevels > len)
            return fail(s, PS_ERR_INVALID, "levels %d..%lld outside the %lld levels of field 1 (LEN)",
                        gts0, (long long)(gts0 - 1 + nlevels), (long long)len);
    }
    PS_CUDA(s, cudaSetDevice(s->device));
    double* dframes = frames;
    const size_t fe = field_elems(s);
    if (frames && !frames_on_device) {
        if (frame_cap > 0) PS_CUDA(s, cudaMallocAsync(&dframes, nbytes(s, (size_t)frame_cap * fe), s->stream));
        else dframes = nullptr;
    }
    int rc;
    if (mode == PS_MODE_SWEPT) rc = run_swept(s, nlevels, gts0, dframes, frame_cap, frame_every);
    else if (mode == PS_MODE_STANDARD) rc = run_standard(s, nlevels, gts0, dframes, frame_cap, frame_every);
    else rc = fail(s, PS_ERR_INVALID, "mode %d", mode);
    if (frames && !frames_on_device && dframes) {
        if (rc == PS_OK)
            PS_CUDA(s, cudaMemcpyAsync(frames, dframes, nbytes(s, (size_t)frame_cap * fe),
                                       cudaMemcpyDeviceToHost, s->stream));
        cudaFreeAsync(dframes, s->stream);
        PS_CUDA(s, cudaStreamSynchronize(s->stream));
    }
    return rc;
}

int ps_get_state(ps_solver* s, double* dst, int level, int dst_on_device)
{
    if (!s || !dst) return PS_ERR_INVALID;
    if (level < 0 || level >= s->its) return fail(s, PS_ERR_INVALID, "level %d not in [0, its)", level);
    PS_CUDA(s, cudaSetDevice(s->device));
    const size_t fe = field_elems(s);
    PS_CUDA(s, cudaMemcpyAsync(dst, at(s, s->base[s->cur], (size_t)(s->its - 1 - level) * fe),
                               nbytes(s, fe),
                               dst_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                               s->stream));
    if (!dst_on_device) PS_CUDA(s, cudaStreamSynchronize(s->stream));
    return PS_OK;
}

// rows [row0, row0+nrows) of every variable of one base level <-> a packed
// [nv][nrows][ny] buffer: one strided copy (variables are nx*ny apart)
static int rows_copy(ps_solver* s, int level, int row0, int nrows, double* buf, int on_device,
                     bool to_buf)
{
    if (!s || !buf) return PS_ERR_INVALID;
    if (level < 0 || level >= s->its) return fail(s, PS_ERR_INVALID, "level %d not in [0, its)", level);
    if (row0 < 0 || nrows < 0 || row0 + nrows > s->nx)
        return fail(s, PS_ERR_INVALID, "rows [%d, %d) outside [0, %d)", row0, row0 + nrows, s->nx);
    if (nrows == 0) return PS_OK;
    PS_CUDA(s, cudaSetDevice(s->device));
    const size_t fe = field_elems(s), plane = (size_t)s->nx * s->ny;
    double* f = at(s, s->base[s->cur], (size_t)(s->its - 1 - level) * fe + (size_t)row0 * s->ny);
    const size_t width = nbytes(s, (size_t)nrows * s->ny);
    if (to_buf)
        PS_CUDA(s, cudaMemcpy2DAsync(buf, width, f, nbytes(s, plane), width, s->nv,
                                     on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                                     s->stream));
    else
        PS_CUDA(s, cudaMemcpy2DAsync(f, nbytes(s, plane), buf, width, width, s->nv,
                                     on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                     s->stream));
    if (!on_device) PS_CUDA(s, cudaStreamSynchronize(s->stream));
    return PS_OK;
}

int ps_get_rows(ps_solver* s, int level, int row0, int nrows, double* dst, int dst_on_device)
{
    return rows_copy(s, level, row0, nrows, dst, dst_on_device, true);
}

int ps_set_rows(ps_solver* s, int level, int row0, int nrows, const double* src, int src_on_device)
{
    if (s && !s->have_state) return fail(s, PS_ERR_STATE, "ps_set_rows before ps_set_state");
    return rows_copy(s, level, row0, nrows, const_cast<double*>(src), src_on_device, false);
}

int ps_synchronize(ps_solver* s)
{
    if (!s) return PS_ERR_INVALID;
    PS_CUDA(s, cudaSetDevice(s->device));
    PS_CUDA(s, cudaStreamSynchronize(s->stream));
    return drain_profile(s);
}

int ps_profile(ps_solver* s, int enable)
{
    if (!s) return PS_ERR_INVALID;
    int rc = ps_synchronize(s);
    if (rc) return rc;
    s->profile = enable != 0;
    for (int i = 0; i < 8; ++i) {
        s->prof_ms[i] = 0;
        s->prof_n[i] = 0;
        s->prof_cells[i] = 0;
    }
    return PS_OK;
}

int ps_profile_read(ps_solver* s, int kind, double* ms, int64_t* launches, double* cells)
{
    if (!s || kind < 0 || kind >= 8) return PS_ERR_INVALID;
    int rc = ps_synchronize(s);
    if (rc) return rc;
    if (ms) *ms = s->prof_ms[kind];
    if (launches) *launches = s->prof_n[kind];
    if (cells) *cells = s->prof_cells[kind];
    return PS_OK;
}

int ps_set_stream(ps_solver* s, void* stream)
{
    if (!s) return PS_ERR_INVALID;
    if (s->own_stream && s->stream) {
        cudaStreamSynchronize(s->stream);
        cudaStreamDestroy(s->stream);
    }
    if (stream) {
        s->stream = (cudaStream_t)stream;
        s->own_stream = false;
    } else {
        PS_CUDA(s, cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
        s->own_stream = true;
    }
    return PS_OK;
}

}  // extern "C"

// ====================================================================== batch
// Many independent instances in one set of launches (include/pysweep_b200.h,
// ps_batch_*).

struct BatchInst {
    int nx = 0, ny = 0, nb = 0, nseg = 1;
    double* base[2] = {nullptr, nullptr};
    double* xface = nullptr;
    double* yface = nullptr;
    size_t yface_n = 0;  // elements of both y-face buffers
    bool have_state = false;
    // levels advanced since this instance's state was set: the step function
    // of the next level sees globalTimeStep = level + 1, as one solver run of
    // all levels so far would show it (the reference starts at 1,
    // pysweep/core/solver.py:162)
    int64_t level = 0;
    std::map<std::string, double> globals;
};

struct ps_batch {
    int device = 0, eq = 0, nv = 1, ops = 1, its = 1, bs = 0, mpss = 0, H = 0;
    int chunk = 32;  // column chunk of the generic streams (32 or 64)
    bool fast = false;
    bool faces = false;  // Euler streams share faces (scratch beside the tile)
    cudaStream_t stream = nullptr;
    // the gap stream runs beside the y-bridge on a high-priority side stream
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    std::vector<BatchInst> inst;
    SweptArgs* d_desc = nullptr;  // [count][2 roles][2 parities] (batch.cuh)
    int2* d_units = nullptr;      // (instance, unit) of every band segment
    int nunits = 0;
    int cur = 0;                  // base holding the current levels (all instances)
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    int64_t graph_levels = -1;
    int graph_cur = -1;
    int64_t graph_launches = 0;
    int64_t launches = 0;
    // the instances' level counters the device descriptors were uploaded with
    std::vector<int64_t> desc_level;
    std::string err;
};

namespace {

int bfail(ps_batch* b, int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (b) b->err = buf;
    else g_create_error = buf;
    return code;
}

#define PSB_CUDA(b, call)                                                                       \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess)                                                                  \
            return bfail((b), e_ == cudaErrorMemoryAllocation ? PS_ERR_NOMEM : PS_ERR_CUDA,     \
                         "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

bool global_allowed(int eq, const char* name)
{
    for (const auto& g : kGlobals)
        if (!strcmp(g.name, name) && (g.eqmask >> eq & 1)) return true;
    return false;
}

void batch_free_graph(ps_batch* b)
{
    if (b->gexec) cudaGraphExecDestroy(b->gexec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->gexec = nullptr;
    b->graph = nullptr;
    b->graph_levels = -1;
}

// Upload both descriptors of every instance (constants may have changed).
int batch_upload(ps_batch* b)
{
    const int n = (int)b->inst.size();
    std::vector<SweptArgs> d(4 * n);
    const int O2 = 2 * b->ops;
    for (int i = 0; i < n; ++i) {
        const BatchInst& I = b->inst[i];
        for (int q = 0; q < 4; ++q) {
            const int role = q / 2, par = q % 2;
            SweptArgs& a = d[4 * i + q];
            memset(&a, 0, sizeof a);
            a.bin = I.base[par];
            a.bout = I.base[1 - par];
            a.xface = I.xface;
            a.yface = I.yface + (role ? I.yface_n / 2 : 0);
            a.frame_every = 1;
            a.nx = I.nx;
            a.ny = I.ny;
            a.nv = b->nv;
            a.bx = b->bs;
            a.hx = b->bs / 2;
            a.Hmax = b->H;
            a.nb = I.nb;
            a.nseg = I.nseg;
            a.wy = I.ny / I.nseg;
            a.nchunks = b->fast ? a.wy / kFastChunk : (a.wy + b->chunk - 1) / b->chunk;
            a.seg_unit = b->fast ? 32 : a.wy;
            a.seg_units = b->fast ? I.ny / 32 : I.nseg;
            a.off = par ? b->bs / 2 : 0;  // prism bands alternate by half a block
            a.its = b->its;
            a.gts_base = (int)I.level;
            a.p = make_params_g(b->eq, I.globals);
            a.seam_direct = seam_direct(b->bs, b->ops, b->nv, b->its, b->H, sizeof(double)) ? 1 : 0;
        }
        (void)O2;
    }
    PSB_CUDA(b, cudaMemcpyAsync(b->d_desc, d.data(), d.size() * sizeof(SweptArgs),
                                cudaMemcpyHostToDevice, b->stream));
    PSB_CUDA(b, cudaStreamSynchronize(b->stream));
    b->desc_level.resize(n);
    for (int i = 0; i < n; ++i) b->desc_level[i] = b->inst[i].level;
    return PS_OK;
}

// Whether the uploaded descriptors carry the instances' current level counters
// (the captured graph reads the descriptors from device memory at every replay).
bool batch_desc_current(const ps_batch* b)
{
    if (b->desc_level.size() != b->inst.size()) return false;
    for (size_t i = 0; i < b->inst.size(); ++i)
        if (b->desc_level[i] != b->inst[i].level) return false;
    return true;
}

size_t batch_tile_smem(const ps_batch* b)
{
    const int O2 = 2 * b->ops, RS = b->chunk + O2;
    return sizeof(double) * ((size_t)(b->its + 1) * b->nv * b->bs * RS +
                             (size_t)(b->H + 1) * b->nv * b->bs * O2);
}

size_t batch_stream_smem(const ps_batch* b)
{
    if (b->fast) return b->bs == 16 ? heat_fast_smem<16>(b->H) : heat_fast_smem<32>(b->H);
    return batch_tile_smem(b) +
           (b->faces ? sizeof(double) * euler_level_scratch(b->bs, b->chunk) : 0);
}

size_t batch_seam_smem(const ps_batch* b)
{
    if (seam_direct(b->bs, b->ops, b->nv, b->its, b->H, sizeof(double)))
        return sizeof(double) * (size_t)(b->its + 1) * b->nv * b->bs * (2 * b->ops * (b->H + 1));
    return sizeof(double) * std::max(seam_smem_elems(false, b->bs, b->ops, b->nv, b->its, b->H),
                                     seam_smem_elems(true, b->bs, b->ops, b->nv, b->its, b->H));
}

using BatchFast = void (*)(const SweptArgs*, const int2*, int, int, int, long long);
using BatchGen = void (*)(const SweptArgs*, const int2*, int, int, long long);

struct BatchKernels {
    const void* P = nullptr;
    const void* G = nullptr;
    const void* Y = nullptr;
    const void* O = nullptr;
};

// Enqueue one half-cycle for every instance: P, then Y on the batch stream
// beside G on the side stream (G reads nothing Y writes; see run_swept), then
// O after both.
template <class Eq, int ITS, int W>
void batch_half(ps_batch* b, int par, int H, long long L0, size_t ssm, size_t gsm, dim3 fgrid)
{
    const int nu = b->nunits;
    cudaStream_t st = b->stream, sd = b->side;
    auto fork = [&] {
        cudaEventRecord(b->ev_fork, st);
        cudaStreamWaitEvent(sd, b->ev_fork, 0);
    };
    auto join = [&] {
        cudaEventRecord(b->ev_join, sd);
        cudaStreamWaitEvent(st, b->ev_join, 0);
    };
    if (b->fast) {
        if (b->bs == 16) {
            heat_stream_fast_batch<16, false><<<fgrid, 32 * kFastWarps, gsm, st>>>(b->d_desc, b->d_units, nu, par, H, L0);
            fork();
            heat_stream_fast_batch<16, true><<<fgrid, 32 * kFastWarps, gsm, sd>>>(b->d_desc, b->d_units, nu, par, H, L0);
        } else {
            heat_stream_fast_batch<32, false><<<fgrid, 32 * kFastWarps, gsm, st>>>(b->d_desc, b->d_units, nu, par, H, L0);
            fork();
            heat_stream_fast_batch<32, true><<<fgrid, 32 * kFastWarps, gsm, sd>>>(b->d_desc, b->d_units, nu, par, H, L0);
        }
    } else {
        stream_batch<Eq, ITS, W, false, 256><<<nu, 256, gsm, st>>>(b->d_desc, b->d_units, par, H, L0);
        fork();
        stream_batch<Eq, ITS, W, true, 256><<<nu, 256, gsm, sd>>>(b->d_desc, b->d_units, par, H, L0);
    }
    if (b->fast) {
        // the register-resident seams, one warp per unit
        const dim3 sgrid((nu + kSeamWarps - 1) / kSeamWarps);
        const size_t ysm =
            (b->bs == 16 ? yseam_smem<16>(b->H) : yseam_smem<32>(b->H)) + kSeamWarps * kDescBytes;
        if (b->bs == 16) {
            heat_seam_fast_batch<16, false><<<sgrid, 32 * kSeamWarps, ysm, st>>>(b->d_desc, b->d_units, nu, par, H, L0);
            join();
            heat_seam_fast_batch<16, true><<<sgrid, 32 * kSeamWarps, ysm, st>>>(b->d_desc, b->d_units, nu, par, H, L0);
        } else {
            heat_seam_fast_batch<32, false><<<sgrid, 32 * kSeamWarps, ysm, st>>>(b->d_desc, b->d_units, nu, par, H, L0);
            join();
            heat_seam_fast_batch<32, true><<<sgrid, 32 * kSeamWarps, ysm, st>>>(b->d_desc, b->d_units, nu, par, H, L0);
        }
        return;
    }
    seam_batch<Eq, ITS, false, 128><<<nu, 128, ssm, st>>>(b->d_desc, b->d_units, par, H, L0);
    join();
    seam_batch<Eq, ITS, true, 128><<<nu, 128, ssm, st>>>(b->d_desc, b->d_units, par, H, L0);
}

template <class Eq, int ITS, int W>
void batch_prepare()
{
    allow_big_smem(heat_stream_fast_batch<16, false>);
    allow_big_smem(heat_stream_fast_batch<16, true>);
    allow_big_smem(heat_stream_fast_batch<32, false>);
    allow_big_smem(heat_stream_fast_batch<32, true>);
    allow_big_smem(heat_seam_fast_batch<16, false>);
    allow_big_smem(heat_seam_fast_batch<16, true>);
    allow_big_smem(heat_seam_fast_batch<32, false>);
    allow_big_smem(heat_seam_fast_batch<32, true>);
    allow_big_smem(stream_batch<Eq, ITS, W, false, 256>);
    allow_big_smem(stream_batch<Eq, ITS, W, true, 256>);
    allow_big_smem(seam_batch<Eq, ITS, false, 128>);
    allow_big_smem(seam_batch<Eq, ITS, true, 128>);
}

using HalfFn = void (*)(ps_batch*, int, int, long long, size_t, size_t, dim3);
using PrepFn = void (*)();

bool batch_pick(int eq, int ops, int its, int chunk, HalfFn* half, PrepFn* prep)
{
#define PS_BSET(EQ, OP, IT, W, T)                                   \
    if (eq == EQ && ops == OP && its == IT && chunk == W) {         \
        *half = batch_half<T, IT, W>;                               \
        *prep = batch_prepare<T, IT, W>;                            \
        return true;                                                \
    }
    PS_BSET(PS_EQ_HEAT, 1, 1, 32, Heat)
    PS_BSET(PS_EQ_HEAT, 1, 2, 32, Heat)
    PS_BSET(PS_EQ_EULER, 2, 2, 32, Euler)
    PS_BSET(PS_EQ_EULER_CELL, 2, 2, 32, EulerCell)
    PS_BSET(PS_EQ_EULER_CELL, 2, 2, 64, EulerCell)
    PS_BSET(PS_EQ_HALF, 1, 2, 32, Half)
#undef PS_BSET
    return false;
}

// Enqueue a whole run of nlevels levels, starting from parity b->cur.
int batch_enqueue(ps_batch* b, int64_t nlevels, HalfFn half, int64_t* nlaunch)
{
    // (the register heat streams' descriptor copies come first in their
    // shared memory)
    const size_t ssm = batch_seam_smem(b),
                 gsm = batch_stream_smem(b) + (b->fast ? kFastWarps * kDescBytes : 0);
    const dim3 fgrid((b->nunits + kFastWarps - 1) / kFastWarps);
    const size_t fe = (size_t)b->nv;
    int par = b->cur;
    int64_t done = 0, n = 0;
    while (done < nlevels) {
        const int H = (int)std::min<int64_t>(b->H, nlevels - done);
        if (H < b->its) {  // the newest its-H base levels carry over unchanged
            for (auto& I : b->inst) {
                const size_t f = fe * I.nx * I.ny;
                for (int q = 0; q < b->its - H; ++q)
                    PSB_CUDA(b, cudaMemcpyAsync(I.base[1 - par] + (size_t)q * f,
                                                I.base[par] + (size_t)(q + H) * f, f * sizeof(double),
                                                cudaMemcpyDeviceToDevice, b->stream));
            }
        }
        half(b, par, H, done, ssm, gsm, fgrid);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return bfail(b, PS_ERR_CUDA, "batched launch: %s", cudaGetErrorString(e));
        n += 4;
        par ^= 1;
        done += H;
    }
    *nlaunch = n;
    return PS_OK;
}

}  // namespace

extern "C" {

int ps_batch_destroy(ps_batch* b);

int ps_batch_create(ps_batch** out, int device, int equation, int count, const int* nx,
                    const int* ny, int nv, int ops, int its, int blocksize)
{
    if (!out || count <= 0 || !nx || !ny) return bfail(nullptr, PS_ERR_INVALID, "bad arguments");
    *out = nullptr;
    HalfFn half;
    PrepFn prep;
    if (!batch_pick(equation, ops, its, 32, &half, &prep))
        return bfail(nullptr, PS_ERR_UNSUPPORTED, "no batched kernels for equation %d ops %d its %d",
                     equation, ops, its);
    if (equation == PS_EQ_EULER && nv != 4) return bfail(nullptr, PS_ERR_INVALID, "euler needs nv=4");
    if ((equation == PS_EQ_HEAT || equation == PS_EQ_HALF) && nv != 1)
        return bfail(nullptr, PS_ERR_INVALID, "heat/half need nv=1");
    if (blocksize % (2 * ops) || blocksize / (2 * ops) - 1 < 1)
        return bfail(nullptr, PS_ERR_INVALID, "blocksize %d invalid for ops %d", blocksize, ops);
    ps_batch* b = new ps_batch();
    b->device = device;
    b->eq = equation;
    b->nv = nv;
    b->ops = ops;
    b->its = its;
    b->bs = blocksize;
    b->mpss = blocksize / (2 * ops) - 1;
    b->H = default_levels(equation, its, blocksize, b->mpss);
    b->fast = equation == PS_EQ_HEAT && its == 1 && (blocksize == 16 || blocksize == 32);
    // Euler: 64-column chunks where the tile fits, faces shared between cells
    // where tile and scratch leave room for two CTAs per SM (as for a solver)
    if (!b->fast && equation == PS_EQ_EULER) {
        b->chunk = 64;
        if (batch_tile_smem(b) > 227 * 1024) b->chunk = 32;
        b->faces = batch_tile_smem(b) + sizeof(double) * euler_level_scratch(b->bs, b->chunk) <=
                   kFaceSmemCap;
    }
    int rc = PS_OK;
    std::vector<int2> units;
    for (int i = 0; i < count && rc == PS_OK; ++i) {
        BatchInst I;
        I.nx = nx[i];
        I.ny = ny[i];
        if (I.nx % blocksize || I.ny % blocksize || (b->fast && I.ny % 32))
            rc = bfail(b, PS_ERR_INVALID, "instance %d: %dx%d not divisible by blocksize %d%s", i,
                       I.nx, I.ny, blocksize, b->fast ? " and 32" : "");
        else if ((size_t)3 * nv * I.nx * I.ny >= (size_t)1 << 31)
            rc = bfail(b, PS_ERR_UNSUPPORTED, "instance %d too large for 32-bit offsets", i);
        else if (!b->fast && 32 < 2 * ops * (b->H + 1))
            rc = bfail(b, PS_ERR_UNSUPPORTED, "blocksize %d too large for the batched streams", blocksize);
        I.nb = I.nx / blocksize;
        // register streams: segments of about 512 columns (measured: 256 heat
        // instances of 128-2048², 1000 steps, 0.998 s at 256 columns, 0.845 s
        // at 512; narrower segments multiply the seam work per cell).  The
        // generic streams: segments of about 256 columns that divide ny and
        // hold a chunk, so that the units of large and small instances take
        // similar times (a phase waits for its slowest unit)
        if (b->fast) {
            I.nseg = std::max(1, I.ny / (8 * kFastChunk));
        } else {
            const int minw = std::max(b->chunk, 2 * ops * (b->H + 1));
            I.nseg = 1;
            for (int q = 2; q <= I.ny / 256 && I.ny / q >= minw; ++q)
                if (I.ny % q == 0) I.nseg = q;
        }
        for (int u = 0; u < I.nb * I.nseg; ++u) units.push_back(make_int2(i, u));
        b->inst.push_back(I);
    }
    if (rc == PS_OK && batch_seam_smem(b) > 227 * 1024)
        rc = bfail(b, PS_ERR_UNSUPPORTED, "seam tile needs %zu bytes of shared memory",
                   batch_seam_smem(b));
    if (rc == PS_OK) {
        cudaError_t e = cudaSetDevice(device);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
        int lo = 0, hi = 0;
        if (e == cudaSuccess) e = cudaDeviceGetStreamPriorityRange(&lo, &hi);
        if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&b->side, cudaStreamNonBlocking, hi);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming);
        if (e != cudaSuccess) rc = bfail(b, PS_ERR_CUDA, "stream: %s", cudaGetErrorString(e));
    }
    const int O2 = 2 * ops, HF = b->H - 1;
    for (auto& I : b->inst) {
        if (rc != PS_OK) break;
        const size_t f = (size_t)nv * I.nx * I.ny;
        const size_t xn = (size_t)I.nb * HF * 2 * nv * O2 * I.ny;
        // two y-face buffers: prism -> y-bridge and gap -> octahedron
        const size_t yn = 2 * (size_t)I.nb * I.nseg * 2 * HF * nv * blocksize * O2;
        I.yface_n = yn;
        cudaError_t e = cudaMalloc(&I.base[0], f * its * sizeof(double));
        if (e == cudaSuccess) e = cudaMalloc(&I.base[1], f * its * sizeof(double));
        if (e == cudaSuccess && xn) e = cudaMalloc(&I.xface, xn * sizeof(double));
        if (e == cudaSuccess && yn) e = cudaMalloc(&I.yface, yn * sizeof(double));
        if (e != cudaSuccess) rc = bfail(b, PS_ERR_NOMEM, "instance buffers: %s", cudaGetErrorString(e));
    }
    if (rc == PS_OK) {
        b->nunits = (int)units.size();
        cudaError_t e = cudaMalloc(&b->d_desc, 4 * b->inst.size() * sizeof(SweptArgs));
        if (e == cudaSuccess) e = cudaMalloc(&b->d_units, units.size() * sizeof(int2));
        if (e == cudaSuccess)
            e = cudaMemcpy(b->d_units, units.data(), units.size() * sizeof(int2), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) rc = bfail(b, PS_ERR_NOMEM, "batch tables: %s", cudaGetErrorString(e));
    }
    // the kernels of the chosen chunk width (prep opts them into large shared memory)
    const int keq = (equation == PS_EQ_EULER && !b->faces) ? PS_EQ_EULER_CELL : equation;
    if (rc == PS_OK && !batch_pick(keq, ops, its, b->chunk, &half, &prep))
        rc = bfail(b, PS_ERR_UNSUPPORTED, "no batched kernels for chunk %d", b->chunk);
    if (rc == PS_OK) prep();
    if (rc != PS_OK) {
        g_create_error = b->err;
        ps_batch_destroy(b);
        return rc;
    }
    *out = b;
    return PS_OK;
}

int ps_batch_destroy(ps_batch* b)
{
    if (!b) return PS_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    batch_free_graph(b);
    for (auto& I : b->inst) {
        for (auto& p : I.base)
            if (p) cudaFree(p);
        if (I.xface) cudaFree(I.xface);
        if (I.yface) cudaFree(I.yface);
    }
    if (b->d_desc) cudaFree(b->d_desc);
    if (b->d_units) cudaFree(b->d_units);
    if (b->side) {
        cudaStreamSynchronize(b->side);
        cudaStreamDestroy(b->side);
    }
    if (b->ev_fork) cudaEventDestroy(b->ev_fork);
    if (b->ev_join) cudaEventDestroy(b->ev_join);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return PS_OK;
}

int ps_batch_set_global(ps_batch* b, int index, const char* name, const void* value, size_t nbytes)
{
    if (!b || !name || !value) return PS_ERR_INVALID;
    if (!global_allowed(b->eq, name)) return bfail(b, PS_ERR_INVALID, "no constant named %s", name);
    if (nbytes != 1 && nbytes != 2 && nbytes != 4 && nbytes != 8)
        return bfail(b, PS_ERR_INVALID, "constant %s: unsupported size %zu", name, nbytes);
    if (index < -1 || index >= (int)b->inst.size()) return bfail(b, PS_ERR_INVALID, "index %d", index);
    const double v = decode_value(value, nbytes);
    for (int i = 0; i < (int)b->inst.size(); ++i)
        if (index == -1 || index == i) b->inst[i].globals[name] = v;
    batch_free_graph(b);  // constants live in the captured descriptors
    return PS_OK;
}

int ps_batch_set_state(ps_batch* b, int index, const double* src, int levels, int src_on_device)
{
    if (!b || !src || index < 0 || index >= (int)b->inst.size()) return PS_ERR_INVALID;
    if (levels != 1 && levels != b->its) return bfail(b, PS_ERR_INVALID, "levels must be 1 or its");
    PSB_CUDA(b, cudaSetDevice(b->device));
    BatchInst& I = b->inst[index];
    const size_t f = (size_t)b->nv * I.nx * I.ny;
    for (int q = 0; q < b->its; ++q)
        PSB_CUDA(b, cudaMemcpyAsync(I.base[b->cur] + (size_t)q * f, src + (size_t)(levels == 1 ? 0 : q) * f,
                                    f * sizeof(double),
                                    src_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                    b->stream));
    if (!src_on_device) PSB_CUDA(b, cudaStreamSynchronize(b->stream));
    I.have_state = true;
    I.level = 0;
    return PS_OK;
}

int ps_batch_run(ps_batch* b, int64_t nlevels, int use_graph)
{
    if (!b) return PS_ERR_INVALID;
    if (nlevels < 0) return bfail(b, PS_ERR_INVALID, "negative level count");
    for (size_t i = 0; i < b->inst.size(); ++i)
        if (!b->inst[i].have_state) return bfail(b, PS_ERR_STATE, "instance %zu has no state", i);
    PSB_CUDA(b, cudaSetDevice(b->device));
    HalfFn half;
    PrepFn prep;
    batch_pick((b->eq == PS_EQ_EULER && !b->faces) ? PS_EQ_EULER_CELL : b->eq, b->ops, b->its,
               b->chunk, &half, &prep);
    const int64_t nhalf = (nlevels + b->H - 1) / b->H;
    if (!use_graph) {
        int rc = batch_upload(b);
        if (rc) return rc;
        int64_t n = 0;
        rc = batch_enqueue(b, nlevels, half, &n);
        if (rc) return rc;
        b->launches += n;
    } else {
        if (!b->gexec || b->graph_levels != nlevels || b->graph_cur != b->cur) {
            batch_free_graph(b);
            int rc = batch_upload(b);
            if (rc) return rc;
            PSB_CUDA(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
            int64_t n = 0;
            rc = batch_enqueue(b, nlevels, half, &n);
            cudaGraph_t g = nullptr;
            cudaError_t e = cudaStreamEndCapture(b->stream, &g);
            if (rc) {
                if (g) cudaGraphDestroy(g);
                return rc;
            }
            if (e != cudaSuccess) return bfail(b, PS_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
            b->graph = g;
            PSB_CUDA(b, cudaGraphInstantiate(&b->gexec, g, 0));
            b->graph_levels = nlevels;
            b->graph_cur = b->cur;
            b->graph_launches = n;
        } else if (!batch_desc_current(b)) {
            int rc = batch_upload(b);  // new level counters for the same graph
            if (rc) return rc;
        }
        PSB_CUDA(b, cudaGraphLaunch(b->gexec, b->stream));
        b->launches += b->graph_launches;
    }
    b->cur ^= (int)(nhalf & 1);
    for (auto& I : b->inst) I.level += nlevels;
    return PS_OK;
}

int ps_batch_get_state(ps_batch* b, int index, double* dst, int level, int dst_on_device)
{
    if (!b || !dst || index < 0 || index >= (int)b->inst.size()) return PS_ERR_INVALID;
    if (level < 0 || level >= b->its) return bfail(b, PS_ERR_INVALID, "level %d", level);
    PSB_CUDA(b, cudaSetDevice(b->device));
    BatchInst& I = b->inst[index];
    const size_t f = (size_t)b->nv * I.nx * I.ny;
    PSB_CUDA(b, cudaMemcpyAsync(dst, I.base[b->cur] + (size_t)(b->its - 1 - level) * f,
                                f * sizeof(double),
                                dst_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                                b->stream));
    if (!dst_on_device) PSB_CUDA(b, cudaStreamSynchronize(b->stream));
    return PS_OK;
}

int ps_batch_synchronize(ps_batch* b)
{
    if (!b) return PS_ERR_INVALID;
    PSB_CUDA(b, cudaSetDevice(b->device));
    PSB_CUDA(b, cudaStreamSynchronize(b->stream));
    return PS_OK;
}

int64_t ps_batch_launches(const ps_batch* b) { return b ? b->launches : 0; }

const char* ps_batch_last_error(const ps_batch* b) { return b ? b->err.c_str() : g_create_error.c_str(); }

int ps_batch_units(const ps_batch* b) { return b ? b->nunits : 0; }

}  // extern "C"
