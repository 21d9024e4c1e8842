// Device vector kernels: FP64 dot products and max-norms with deterministic two-stage
// reductions (fixed grid, fixed summation order), the initial guess, and the L-BFGS
// buffers (the minimiser's own passes are in k_lbfgs.cuh).
#pragma once

#include "common.cuh"

namespace mdft {

constexpr int kRedBlocks = 1184;  // 8 x 148 SMs, fixed so that sums are reproducible
constexpr int kRedThreads = 256;

// part[blk*2+0] = sum a*b, part[blk*2+1] = max |a|  (b may be null -> sum a*a)
__global__ void __launch_bounds__(kRedThreads) k_dot_max(const double *__restrict__ a, const double *__restrict__ b,
                                                         long long n, double *__restrict__ part) {
    double s = 0.0, mx = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        double x = a[i];
        s = fma(x, b ? b[i] : x, s);
        mx = fmax(mx, fabs(x));
    }
    __shared__ double ss[kRedThreads / 32], sm[kRedThreads / 32];
    for (int off = 16; off > 0; off >>= 1) {
        s += __shfl_down_sync(0xffffffffu, s, off);
        mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, off));
    }
    if ((threadIdx.x & 31) == 0) {
        ss[threadIdx.x >> 5] = s;
        sm[threadIdx.x >> 5] = mx;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0, u = 0.0;
        for (int i = 0; i < kRedThreads / 32; ++i) {
            t += ss[i];
            u = fmax(u, sm[i]);
        }
        part[2 * blockIdx.x + 0] = t;
        part[2 * blockIdx.x + 1] = u;
    }
}

// out[slot] = sum of part[.,0], out[slot+1] = max of part[.,1]
__global__ void k_finish_dot_max(const double *__restrict__ part, int nblk, double *__restrict__ out, int slot) {
    __shared__ double ss[256], sm[256];
    double s = 0.0, mx = 0.0;
    for (int i = threadIdx.x; i < nblk; i += blockDim.x) {
        s += part[2 * i];
        mx = fmax(mx, part[2 * i + 1]);
    }
    ss[threadIdx.x] = s;
    sm[threadIdx.x] = mx;
    __syncthreads();
    for (int off = blockDim.x / 2; off > 0; off >>= 1) {
        if ((int)threadIdx.x < off) {
            ss[threadIdx.x] += ss[threadIdx.x + off];
            sm[threadIdx.x] = fmax(sm[threadIdx.x], sm[threadIdx.x + off]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[slot] = ss[0];
        out[slot + 1] = sm[0];
    }
}

// xi = vext >= vmax ? 0 : 1   (guess_density, src/module_density.f90:267-284)
__global__ void k_guess(const double *__restrict__ vext, double *__restrict__ xi, double vmax, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        xi[i] = (vext[i] >= vmax) ? 0.0 : 1.0;
}

struct LbfgsState {
    long long n = 0;
    int m = 0;
    DevBuf<double> x, d, t, r, S, Y;  // point, direction, trial point, trial gradient, history
};

inline void lbfgs_free(LbfgsState &s) {
    s.x.free(); s.d.free(); s.t.free(); s.r.free(); s.S.free(); s.Y.free();
    s.n = 0;
    s.m = 0;
}

constexpr int kScalarSlots = 512;  // device scalars of the vector reductions

}  // namespace mdft
