// Device vector kernels of the L-BFGS driver: FP64 dot products and max-norms
// with deterministic two-stage reductions (fixed grid, fixed summation
// order), and the element-wise updates of src/module_lbfgs_nocedal_mdft.f90.
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

// y = a - b (into y), partial sums of y*y
__global__ void __launch_bounds__(kRedThreads) k_diff_norm(const double *__restrict__ a, double *__restrict__ y, long long n,
                                                           double *__restrict__ part) {
    double s = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        double v = a[i] - y[i];
        y[i] = v;
        s = fma(v, v, s);
    }
    __shared__ double ss[kRedThreads / 32];
    for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
    if ((threadIdx.x & 31) == 0) ss[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int i = 0; i < kRedThreads / 32; ++i) t += ss[i];
        part[2 * blockIdx.x] = t;
        part[2 * blockIdx.x + 1] = 0.0;
    }
}

// z = x - g ; d = z - x   (generalised Cauchy point with no bounds and theta = 1)
__global__ void k_sd_step(const double *__restrict__ x, const double *__restrict__ g, double *__restrict__ z,
                          double *__restrict__ d, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        double zi = x[i] - g[i];
        z[i] = zi;
        d[i] = zi - x[i];
    }
}

// z = x + q ; d = z - x
__global__ void k_qn_step(const double *__restrict__ x, const double *__restrict__ q, double *__restrict__ z,
                          double *__restrict__ d, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        double zi = x[i] + q[i];
        z[i] = zi;
        d[i] = zi - x[i];
    }
}

// q = -g
__global__ void k_neg(const double *__restrict__ g, double *__restrict__ q, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) q[i] = -g[i];
}

// Two-loop recursion step: q += coef * v, coef = sgn * rho * sc[slot] (+ extra), and
// partial dot of the updated q with w (w may be null).
__global__ void __launch_bounds__(kRedThreads) k_axpy_dot(double *__restrict__ q, const double *__restrict__ v,
                                                          const double *__restrict__ w, long long n,
                                                          const double *__restrict__ sc, int slot_a, double rho_a,
                                                          int slot_b, double rho_b, double scale,
                                                          double *__restrict__ part) {
    // coef = rho_a*sc[slot_a] - rho_b*sc[slot_b]   (slot < 0 -> term absent); q = scale*q + coef*v
    double coef = 0.0;
    if (slot_a >= 0) coef += rho_a * sc[slot_a];
    if (slot_b >= 0) coef -= rho_b * sc[slot_b];
    double s = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        double qi = scale * q[i];
        if (v) qi = fma(coef, v[i], qi);
        q[i] = qi;
        if (w) s = fma(qi, w[i], s);
    }
    if (!part) return;
    __shared__ double ss[kRedThreads / 32];
    for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
    if ((threadIdx.x & 31) == 0) ss[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int i = 0; i < kRedThreads / 32; ++i) t += ss[i];
        part[2 * blockIdx.x] = t;
        part[2 * blockIdx.x + 1] = 0.0;
    }
}

// x = (stp == 1) ? z : stp * d + t     (src/module_lbfgs_nocedal_mdft.f90 lnsrlb)
__global__ void k_trial_point(double *__restrict__ x, const double *__restrict__ z, const double *__restrict__ d,
                              const double *__restrict__ t, double stp, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        x[i] = (stp == 1.0) ? z[i] : fma(stp, d[i], t[i]);
}

// s = stp * d (or d when stp == 1)
__global__ void k_scale_copy(double *__restrict__ s, const double *__restrict__ d, double stp, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        s[i] = (stp == 1.0) ? d[i] : stp * d[i];
}

// xi = vext >= vmax ? 0 : 1   (guess_density, src/module_density.f90:267-284)
__global__ void k_guess(const double *__restrict__ vext, double *__restrict__ xi, double vmax, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        xi[i] = (vext[i] >= vmax) ? 0.0 : 1.0;
}

struct LbfgsState {
    long long n = 0;
    int m = 0;
    DevBuf<double> x, z, d, t, r, q, S, Y;
};

inline void lbfgs_free(LbfgsState &s) {
    s.x.free(); s.z.free(); s.d.free(); s.t.free(); s.r.free(); s.q.free(); s.S.free(); s.Y.free();
    s.n = 0;
    s.m = 0;
}

constexpr int kScalarSlots = 512;  // device scalars of the vector reductions

}  // namespace mdft
