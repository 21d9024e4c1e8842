// Ideal + external term with no device allocation: the per-block partial sums
// live in a fixed array inside the library instead of a buffer from cudaMalloc.
#include "../../include/mdft_b200.h"

#include <mutex>

#include <cuda.h>
#include <cuda_runtime.h>

#include "common.cuh"

namespace {

constexpr int kPointsPerBlock = 64;
constexpr int kThreads = 256;
constexpr int kMaxBlocks = 16384;  // => at most 1,048,576 grid points per call
constexpr int kMaxDevices = 64;
constexpr double kEpsDp = 2.220446049250313080847263336181640625e-16;

// Partial sums {F_id, F_ext} of every block of the last call (256 KB on every GPU that
// loads the library, kept until the process exits).  Each call overwrites the entries it
// reads back, so nothing carries over between calls; calls that overlap on the GPU race.
static __device__ __align__(256) double g_partials[2 * kMaxBlocks];

// Device address of g_partials per device, looked up on the first call on that device and
// again whenever the current context is not the one it was looked up in: cudaDeviceReset
// destroys the primary context, and the array may sit elsewhere in the next one.
struct ScratchSlot {
    double *addr = nullptr;
    unsigned long long ctx_id = 0;  // unique id of the context the address belongs to
};
ScratchSlot g_slots[kMaxDevices];
std::mutex g_lock;

// Unique id of the calling thread's current context (cuCtxGetCurrent + cuCtxGetId, reached
// through the runtime's driver entry points so that the library needs no libcuda link).
// false when no context is current or the driver does not offer the query.
bool current_context_id(unsigned long long *id) {
    using GetCurrentFn = CUresult (*)(CUcontext *);
    using GetIdFn = CUresult (*)(CUcontext, unsigned long long *);
    static GetCurrentFn get_current = nullptr;
    static GetIdFn get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *a = nullptr, *b = nullptr;
        cudaDriverEntryPointQueryResult qa{}, qb{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa) == cudaSuccess &&
            qa == cudaDriverEntryPointSuccess &&
            cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb) == cudaSuccess &&
            qb == cudaDriverEntryPointSuccess) {
            get_current = reinterpret_cast<GetCurrentFn>(a);
            get_id = reinterpret_cast<GetIdFn>(b);
        }
        cudaGetLastError();
    });
    if (!get_current || !get_id) return false;
    CUcontext ctx = nullptr;
    if (get_current(&ctx) != CUDA_SUCCESS || !ctx) return false;
    return get_id(ctx, id) == CUDA_SUCCESS;
}

// energy_ideal_and_external (src/module_energy_ideal_and_external.f90:46-73) over the
// points [blockIdx.x*64, +64) of one block: partial F_id, F_ext and df = id+ext gradient.
__global__ void __launch_bounds__(kThreads) k_ideal_external_partials(const double *__restrict__ xi, const double *__restrict__ vext,
                                                                    const double *__restrict__ w, int no, long long npoints,
                                                                    double kT, double rho0, double dv, double *__restrict__ df,
                                                                    double *__restrict__ partials) {
    const long long first = (long long)blockIdx.x * kPointsPerBlock * no;
    const long long last = min(first + (long long)kPointsPerBlock * no, npoints * no);
    double fid = 0.0, fext = 0.0;
    for (long long i = first + threadIdx.x; i < last; i += blockDim.x) {
        const int io = (int)(i % no);
        const double x = xi[i], wio = w[io];
        const double rho = x * x * rho0;
        double g = 0.0;
        if (rho > kEpsDp) {
            const double lg = log(rho / rho0), v = vext[i];
            fid += kT * dv * wio * (rho * lg - rho + rho0);
            fext += dv * wio * rho * v;
            g = wio * 2.0 * rho0 * x * (kT * lg + v);
        } else {
            fid += kT * dv * wio * rho0;
        }
        if (df) df[i] = g;
    }
    __shared__ double s_id[kThreads / 32], s_ext[kThreads / 32];
    for (int off = 16; off > 0; off >>= 1) {
        fid += __shfl_down_sync(0xffffffffu, fid, off);
        fext += __shfl_down_sync(0xffffffffu, fext, off);
    }
    if ((threadIdx.x & 31) == 0) {
        s_id[threadIdx.x >> 5] = fid;
        s_ext[threadIdx.x >> 5] = fext;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int k = 0; k < kThreads / 32; ++k) {
            a += s_id[k];
            b += s_ext[k];
        }
        partials[2 * blockIdx.x] = a;
        partials[2 * blockIdx.x + 1] = b;
    }
}

// Sum the nblk partial pairs in a fixed order into out[0..1].
__global__ void k_sum_partials(const double *__restrict__ partials, int nblk, double *__restrict__ out) {
    __shared__ double sa[kThreads], sb[kThreads];
    double a = 0.0, b = 0.0;
    for (int k = threadIdx.x; k < nblk; k += blockDim.x) {
        a += partials[2 * k];
        b += partials[2 * k + 1];
    }
    sa[threadIdx.x] = a;
    sb[threadIdx.x] = b;
    __syncthreads();
    for (int off = blockDim.x / 2; off > 0; off >>= 1) {
        if ((int)threadIdx.x < off) {
            sa[threadIdx.x] += sa[threadIdx.x + off];
            sb[threadIdx.x] += sb[threadIdx.x + off];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = sa[0];
        out[1] = sb[0];
    }
}

int fail(int code, const char *msg) {
    mdft::set_error("%s", msg);
    return code;
}

}  // namespace

extern "C" int mdft_ideal_external_noalloc(const double *d_xi, const double *d_vext, const double *d_w, int no,
                                           long long npoints, double kT, double rho0, double dv, double *d_df,
                                           double *d_out, void *stream) {
    if (!d_xi || !d_vext || !d_w || !d_out || no <= 0 || npoints <= 0)
        return fail(MDFT_E_ARG, "mdft_ideal_external_noalloc: null pointer or non-positive size");
    const long long nblk = (npoints + kPointsPerBlock - 1) / kPointsPerBlock;
    if (nblk > kMaxBlocks) {
        mdft::set_error("mdft_ideal_external_noalloc: %lld grid points exceed the fixed scratch limit of %d points",
                        npoints, kMaxBlocks * kPointsPerBlock);
        return MDFT_E_ARG;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(MDFT_E_CUDA, cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return fail(MDFT_E_ARG, "mdft_ideal_external_noalloc: device ordinal out of range");
    double *scratch;
    {
        // First call on this device (or first in a new context): look up the device address
        // of the fixed array (host code may not use &g_partials, which is only a host-side
        // stand-in for it).
        std::lock_guard<std::mutex> lk(g_lock);
        ScratchSlot &slot = g_slots[dev];
        unsigned long long id = 0;
        const bool have_id = current_context_id(&id);
        if (!slot.addr || !have_id || id != slot.ctx_id) {
            void *p = nullptr;
            e = cudaGetSymbolAddress(&p, g_partials);
            if (e != cudaSuccess) return fail(MDFT_E_CUDA, cudaGetErrorString(e));
            slot.addr = static_cast<double *>(p);
            // the lookup made the device's context current if none was
            slot.ctx_id = current_context_id(&id) ? id : 0;
            if (!slot.ctx_id) slot.addr = nullptr;  // no id to check against: look up on every call
            scratch = static_cast<double *>(p);
        } else {
            scratch = slot.addr;
        }
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    k_ideal_external_partials<<<(unsigned)nblk, kThreads, 0, st>>>(d_xi, d_vext, d_w, no, npoints, kT, rho0, dv, d_df, scratch);
    k_sum_partials<<<1, kThreads, 0, st>>>(scratch, (int)nblk, d_out);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(MDFT_E_CUDA, cudaGetErrorString(e));
    return MDFT_OK;
}
