// Batched 3-D complex FFTs over every projection plane (S2/S6 of
// src/module_energy_cproj_mrso.f90:306-329,690-719), written for this engine:
// one kernel per axis; a CTA stages a tile of TL lines (TL consecutive x for
// the y and z axes, TL consecutive rows for the x axis, so every global access
// is coalesced) in shared memory and runs a mixed-radix (4, 2, 3) Stockham
// transform there.  sign=+1 computes X[k] = sum_j x[j] e^{+2 pi i jk/n} (the
// reference's plan3dp), sign=-1 the plan3dm direction; no scaling.
#pragma once

#include "common.cuh"

namespace mdft {

template <typename T> struct Cplx;
template <> struct Cplx<double> { using t = double2; };
template <> struct Cplx<float> { using t = float2; };

template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
    C r;
    r.x = a.x * b.x - a.y * b.y;
    r.y = a.x * b.y + a.y * b.x;
    return r;
}
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { C r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { C r; r.x = a.x - b.x; r.y = a.y - b.y; return r; }
template <typename C> __device__ __forceinline__ C cconj(C a) { a.y = -a.y; return a; }

constexpr int kFftMaxPass = 10;
constexpr int kFftThreads = 256;

struct FftPlan1D {
    int n = 0;
    int npass = 0;
    int rad[kFftMaxPass] = {0};
};

inline bool make_plan1d(int n, FftPlan1D &p) {
    p.n = n;
    p.npass = 0;
    int r = n;
    while (r % 4 == 0) { p.rad[p.npass++] = 4; r /= 4; }
    while (r % 2 == 0) { p.rad[p.npass++] = 2; r /= 2; }
    while (r % 3 == 0) { p.rad[p.npass++] = 3; r /= 3; }
    return r == 1 && p.npass <= kFftMaxPass;
}

struct FftAxisArgs {
    int axis;  // 0 = x, 1 = y, 2 = z
    int nx, ny, nz;
    long long nplanes;
    int TL;     // lines per tile
    int sign;   // +1 or -1
    FftPlan1D plan;
};

template <typename T>
__global__ void __launch_bounds__(kFftThreads) k_fft_axis(typename Cplx<T>::t *__restrict__ data,
                                                          const typename Cplx<T>::t *__restrict__ tw, FftAxisArgs a) {
    using C = typename Cplx<T>::t;
    extern __shared__ unsigned char fft_smem_raw[];
    C *buf0 = reinterpret_cast<C *>(fft_smem_raw);
    const int n = a.plan.n, TL = a.TL, LD = TL + 1;
    C *buf1 = buf0 + (size_t)n * LD;
    // tile -> base offset and strides
    const long long plane = (long long)a.nx * a.ny * a.nz;
    long long base;
    long long istride, lstride;
    long long t = blockIdx.x;
    if (a.axis == 0) {
        istride = 1;
        lstride = a.nx;
        base = t * TL * (long long)a.nx;
    } else {
        const int xt = a.nx / TL;
        const long long ix0 = (t % xt) * TL;
        const long long rest = t / xt;
        lstride = 1;
        if (a.axis == 1) {
            istride = a.nx;
            base = rest * (long long)a.ny * a.nx + ix0;  // rest = p*nz + iz
        } else {
            istride = (long long)a.nx * a.ny;
            const long long p = rest / a.ny, iy = rest % a.ny;
            base = p * plane + iy * a.nx + ix0;
        }
    }
    // load
    for (int f = threadIdx.x; f < n * TL; f += blockDim.x) {
        int i, l;
        if (a.axis == 0) { i = f % n; l = f / n; }
        else { i = f / TL; l = f % TL; }
        buf0[i * LD + l] = data[base + i * istride + l * lstride];
    }
    __syncthreads();
    C *in = buf0, *out = buf1;
    int Ns = 1;
    for (int ps = 0; ps < a.plan.npass; ++ps) {
        const int R = a.plan.rad[ps];
        const int nb = n / R;
        const int tstep = n / (Ns * R);
        for (int it = threadIdx.x; it < nb * TL; it += blockDim.x) {
            const int j = it / TL, l = it % TL;
            const int jm = j % Ns;
            C v[4];
            for (int r = 0; r < R; ++r) {
                C x = in[(j + r * nb) * LD + l];
                if (r > 0 && jm > 0) {
                    C w = tw[(jm * tstep * r) % n];
                    if (a.sign < 0) w = cconj(w);
                    x = cmul(x, w);
                }
                v[r] = x;
            }
            C y[4];
            if (R == 2) {
                y[0] = cadd(v[0], v[1]);
                y[1] = csub(v[0], v[1]);
            } else if (R == 4) {
                C s02 = cadd(v[0], v[2]), d02 = csub(v[0], v[2]);
                C s13 = cadd(v[1], v[3]), d13 = csub(v[1], v[3]);
                // w = sign * i ; w * d13
                C wd;
                wd.x = -a.sign * d13.y;
                wd.y = a.sign * d13.x;
                y[0] = cadd(s02, s13);
                y[1] = cadd(d02, wd);
                y[2] = csub(s02, s13);
                y[3] = csub(d02, wd);
            } else {  // R == 3
                const T c3 = (T)-0.5;
                const T s3 = (T)(a.sign * 0.86602540378443864676372317075294);
                C s12 = cadd(v[1], v[2]), d12 = csub(v[1], v[2]);
                C m;
                m.x = v[0].x + c3 * s12.x;
                m.y = v[0].y + c3 * s12.y;
                C rot;  // i * s3 * d12
                rot.x = -s3 * d12.y;
                rot.y = s3 * d12.x;
                y[0] = cadd(v[0], s12);
                y[1] = cadd(m, rot);
                y[2] = csub(m, rot);
            }
            const int idxD = (j / Ns) * Ns * R + jm;
            for (int r = 0; r < R; ++r) out[(idxD + r * Ns) * LD + l] = y[r];
        }
        __syncthreads();
        C *tmp = in;
        in = out;
        out = tmp;
        Ns *= R;
    }
    for (int f = threadIdx.x; f < n * TL; f += blockDim.x) {
        int i, l;
        if (a.axis == 0) { i = f % n; l = f / n; }
        else { i = f / TL; l = f % TL; }
        data[base + i * istride + l * lstride] = in[i * LD + l];
    }
}

template <typename T>
inline size_t fft_smem_bytes(int n, int TL) {
    return 2 * sizeof(typename Cplx<T>::t) * (size_t)n * (TL + 1);
}

}  // namespace mdft
