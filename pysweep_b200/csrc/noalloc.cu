// ps_heat_swept_noalloc: the swept heat path for callers that cannot allocate
// device memory.
//
// Some hosts of this library run where a cudaMalloc is not allowed at call
// time: plugins of a process whose memory pool owns the whole device, or
// real-time loops that must not touch the allocator.  This entry point takes
// only the caller's input and output fields and keeps every temporary buffer
// in one file-scope device array, g_noalloc_scratch, that the CUDA runtime
// reserves on each device when the library is loaded.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/pysweep_b200.h"
#include "heat_fast.cuh"
#include "seam_fast.cuh"
#include "swept.cuh"

namespace {

// Scratch for one call: an intermediate field plus the prism faces.  Held by
// every GPU that loads the library, for the life of the process.
constexpr size_t kScratchBytes = (size_t)128 << 20;  // 128 MiB
__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_ptr[kMaxDevices] = {};

void put_err(char* err, size_t errlen, const char* msg)
{
    if (err && errlen) {
        strncpy(err, msg, errlen - 1);
        err[errlen - 1] = '\0';
    }
}

size_t round_up(size_t v) { return (v + 255) & ~(size_t)255; }

// Whether the byte ranges [a, a+na) and [b, b+nb) share a byte.
bool overlap(const void* a, size_t na, const void* b, size_t nb)
{
    const uintptr_t x = (uintptr_t)a, y = (uintptr_t)b;
    return x < y + nb && y < x + na;
}

}  // namespace

using namespace psb;

extern "C" int ps_heat_swept_noalloc(const double* d_in, double* d_out, int nx, int ny,
                                     int blocksize, int64_t nsteps, double alpha, double dt,
                                     double dx, void* stream, char* err, size_t errlen)
{
    char msg[256];
    if (!d_in || !d_out) {
        put_err(err, errlen, "d_in and d_out must be device pointers");
        return PS_ERR_INVALID;
    }
    if ((blocksize != 16 && blocksize != 32) || nx <= 0 || ny <= 0 || nx % blocksize ||
        ny % kFastChunk || nsteps < 0) {
        snprintf(msg, sizeof msg,
                 "need blocksize 16 or 32, nx a multiple of it, ny a multiple of %d, nsteps >= 0 "
                 "(got bs %d, %dx%d, %lld steps)",
                 kFastChunk, blocksize, nx, ny, (long long)nsteps);
        put_err(err, errlen, msg);
        return PS_ERR_INVALID;
    }
    cudaStream_t st = (cudaStream_t)stream;
    const size_t fe = (size_t)nx * ny;
    // tiling: the defaults of a ps_solver (MPSS levels per half-cycle, one
    // wave of warps); results do not depend on it
    int dev = 0;
    cudaGetDevice(&dev);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int BX = blocksize, H = BX / 2 - 1, HF = H - 1, nb = nx / BX;
    const int nseg =
        std::max(1, std::min(ny / kFastChunk, sms * fast_ctas_per_sm(BX, 0) * kFastWarps / nb));
    const size_t field_b = round_up(fe * sizeof(double));
    const size_t xface_b = round_up((size_t)nb * HF * 2 * 2 * ny * sizeof(double));
    const size_t yface_b = round_up((size_t)nb * nseg * 2 * HF * BX * 2 * sizeof(double));
    const size_t need = field_b + xface_b + yface_b;
    if (need > kScratchBytes) {
        snprintf(msg, sizeof msg,
                 "%dx%d with blocksize %d needs %zu bytes of scratch; the built-in scratch "
                 "holds %zu bytes",
                 nx, ny, blocksize, need, kScratchBytes);
        put_err(err, errlen, msg);
        return PS_ERR_INVALID;
    }
    if (overlap(d_in, fe * sizeof(double), d_out, fe * sizeof(double))) {
        put_err(err, errlen, "d_in and d_out overlap: the solve reads d_in while it writes d_out");
        return PS_ERR_INVALID;
    }
    if (nsteps == 0) {
        cudaError_t e = cudaMemcpyAsync(d_out, d_in, fe * sizeof(double),
                                        cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) {
            put_err(err, errlen, cudaGetErrorString(e));
            return PS_ERR_CUDA;
        }
        return PS_OK;
    }
    if (dev < 0 || dev >= kMaxDevices) {
        put_err(err, errlen, "device ordinal out of range");
        return PS_ERR_INVALID;
    }
    // set-up, once per device: the device address of the scratch array (the
    // host-side symbol is not a device address)
    void* base = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_mu);
        if (!g_scratch_ptr[dev]) {
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p) {
                snprintf(msg, sizeof msg, "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
                put_err(err, errlen, msg);
                return PS_ERR_CUDA;
            }
            const void* kernels[] = {
                (const void*)heat_stream_fast<16, false>, (const void*)heat_stream_fast<16, true>,
                (const void*)heat_stream_fast<32, false>, (const void*)heat_stream_fast<32, true>,
                (const void*)heat_yseam_fast<16>, (const void*)heat_oseam_fast<16>,
                (const void*)heat_yseam_fast<32>, (const void*)heat_oseam_fast<32>};
            for (const void* k : kernels) {
                e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
                if (e != cudaSuccess) {
                    snprintf(msg, sizeof msg, "cudaFuncSetAttribute: %s", cudaGetErrorString(e));
                    put_err(err, errlen, msg);
                    return PS_ERR_CUDA;  // the device stays unset: the next call retries
                }
            }
            g_scratch_ptr[dev] = p;
        }
        base = g_scratch_ptr[dev];
    }
    if (overlap(d_in, fe * sizeof(double), base, need) ||
        overlap(d_out, fe * sizeof(double), base, need)) {
        put_err(err, errlen, "d_in or d_out lies inside the library's scratch array");
        return PS_ERR_INVALID;
    }
    double* A = (double*)base;
    SweptArgs a;
    memset(&a, 0, sizeof a);
    a.nx = nx;
    a.ny = ny;
    a.nv = 1;
    a.bx = BX;
    a.hx = BX / 2;
    a.Hmax = H;
    a.nb = nb;
    a.nseg = nseg;
    a.wy = ny / nseg;
    a.nchunks = a.wy / kFastChunk;
    a.seg_unit = 32;
    a.seg_units = ny / 32;
    a.its = 1;
    a.gts_base = 0;
    a.frame_every = 1;
    a.xface = (double*)((unsigned char*)base + field_b);
    a.yface = (double*)((unsigned char*)base + field_b + xface_b);
    a.p.d[0] = alpha * dt / dx / dx;  // heat.py:37
    a.p.i[0] = 1;                     // forward Euler
    const int units = nb * nseg;
    const int fgrid = (units + kFastWarps - 1) / kFastWarps;
    const size_t fsm = BX == 16 ? heat_fast_smem<16>(H) : heat_fast_smem<32>(H);
    // the register seams: one warp per block edge
    const int sgrid = (units + kSeamWarps - 1) / kSeamWarps;
    const size_t ssm = BX == 16 ? yseam_smem<16>(H) : yseam_smem<32>(H);
    const int64_t halves = (nsteps + H - 1) / H;
    // outputs alternate between d_out and the scratch field so that the last
    // half-cycle lands in d_out and d_in is only read
    const double* in = d_in;
    int64_t done = 0;
    int off = 0;
    for (int64_t t = 0; t < halves; ++t) {
        const int h = (int)std::min<int64_t>(H, nsteps - done);
        double* out = ((halves - 1 - t) % 2 == 0) ? d_out : A;
        a.H = h;
        a.L0 = done;
        a.off = off;
        a.bin = in;
        a.bout = out;
        if (BX == 16) {
            heat_stream_fast<16, false><<<fgrid, 32 * kFastWarps, fsm, st>>>(a);
            heat_yseam_fast<16><<<sgrid, 32 * kSeamWarps, ssm, st>>>(a);
            heat_stream_fast<16, true><<<fgrid, 32 * kFastWarps, fsm, st>>>(a);
            heat_oseam_fast<16><<<sgrid, 32 * kSeamWarps, ssm, st>>>(a);
        } else {
            heat_stream_fast<32, false><<<fgrid, 32 * kFastWarps, fsm, st>>>(a);
            heat_yseam_fast<32><<<sgrid, 32 * kSeamWarps, ssm, st>>>(a);
            heat_stream_fast<32, true><<<fgrid, 32 * kFastWarps, fsm, st>>>(a);
            heat_oseam_fast<32><<<sgrid, 32 * kSeamWarps, ssm, st>>>(a);
        }
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) {
            snprintf(msg, sizeof msg, "kernel launch: %s", cudaGetErrorString(e));
            put_err(err, errlen, msg);
            return PS_ERR_CUDA;
        }
        in = out;
        off = ((off - BX / 2) % nx + nx) % nx;
        done += h;
    }
    return PS_OK;
}
