// Vector passes of the limited-memory BFGS driver in compact form.
//
// The search direction -H g of src/module_lbfgs_nocedal_mdft.f90 (formk/cmprlb/subsm with
// no bounds) is formed as  d = cg g + sum_i a_i s_i + sum_i b_i y_i  with the 2m+1
// coefficients computed on the host from small Gram matrices (Byrd, Nocedal and Schnabel,
// Math. Prog. 63 (1994), eq. 3.1 in inverse form).  A step therefore reads each history
// vector twice -- once for its inner products with the new gradient (k_pair_dots, which also
// forms and stores the new pair), once for the combination (k_direction) -- instead of the
// four passes per pair of the two-loop recursion.
//
// Every reduction is two-stage with the fixed grid kRedBlocks and a fixed summation order,
// so results are reproducible run to run.
#pragma once

#include "common.cuh"
#include "k_vec.cuh"

namespace mdft {

constexpr int kPairGroup = 8;    // history slots read per k_pair_dots launch
constexpr int kMaxRows = 4 * kPairGroup + 4;  // reduction rows of one launch

// MODE 0: rows s_i.g [0,K), y_i.g [K,2K), g.g [2K]
// MODE 1: forms s_new = stp d and y_new = g - gold (stored), rows as MODE 0 plus
//         s_i.y_new [2K+1,3K+1), y_i.y_new [3K+1,4K+1), y_new.y_new, y_new.g, s_new.g
// MODE 2: y_new read back from ynew; rows as MODE 1 without the last three
struct PairDotsArgs {
    const double *g, *gold, *d;
    const double *s[kPairGroup], *y[kPairGroup];
    double *snew, *ynew;
    double stp;
    long long n;
    double *part;  // [rows][gridDim.x]
};

template <int K, int MODE> __host__ __device__ constexpr int pair_rows() {
    return MODE == 0 ? 2 * K + 1 : (MODE == 1 ? 4 * K + 4 : 4 * K + 1);
}

template <int R>
__device__ __forceinline__ void block_rows_store(double (&acc)[R], double *part) {
    __shared__ double red[kMaxRows][kRedThreads / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        double v = acc[r];
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        if (lane == 0) red[r][wid] = v;
    }
    __syncthreads();
    if ((int)threadIdx.x < R) {
        double t = 0.0;
        for (int i = 0; i < kRedThreads / 32; ++i) t += red[threadIdx.x][i];
        part[(size_t)threadIdx.x * gridDim.x + blockIdx.x] = t;
    }
}

template <int K, int MODE>
__global__ void __launch_bounds__(kRedThreads) k_pair_dots(PairDotsArgs a) {
    constexpr int R = pair_rows<K, MODE>();
    double acc[R];
#pragma unroll
    for (int r = 0; r < R; ++r) acc[r] = 0.0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
        const double gi = a.g[i];
        double yn = 0.0;
        if constexpr (MODE == 1) {
            yn = gi - a.gold[i];
            const double sn = (a.stp == 1.0) ? a.d[i] : a.stp * a.d[i];
            a.snew[i] = sn;
            a.ynew[i] = yn;
            acc[4 * K + 1] = fma(yn, yn, acc[4 * K + 1]);
            acc[4 * K + 2] = fma(yn, gi, acc[4 * K + 2]);
            acc[4 * K + 3] = fma(sn, gi, acc[4 * K + 3]);
        } else if constexpr (MODE == 2) {
            yn = a.ynew[i];
        }
        acc[2 * K] = fma(gi, gi, acc[2 * K]);
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const double si = a.s[k][i], yi = a.y[k][i];
            acc[k] = fma(si, gi, acc[k]);
            acc[K + k] = fma(yi, gi, acc[K + k]);
            if constexpr (MODE != 0) {
                acc[2 * K + 1 + k] = fma(si, yn, acc[2 * K + 1 + k]);
                acc[3 * K + 1 + k] = fma(yi, yn, acc[3 * K + 1 + k]);
            }
        }
    }
    block_rows_store<R>(acc, a.part);
}

// d = (accumulate ? d : cg g) + sum_k cv_k v_k ; with part: rows g.d, d.d
struct DirArgs {
    const double *g;
    double cg;
    const double *v[2 * kPairGroup];
    double cv[2 * kPairGroup];
    double *d;
    int accumulate;
    long long n;
    double *part;
};

template <int K>
__global__ void __launch_bounds__(kRedThreads) k_direction(DirArgs a) {
    double acc[2] = {0.0, 0.0};
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
        const bool need_g = !a.accumulate || a.part;
        const double gi = need_g ? a.g[i] : 0.0;
        double di = a.accumulate ? a.d[i] : a.cg * gi;
#pragma unroll
        for (int k = 0; k < K; ++k) di = fma(a.cv[k], a.v[k][i], di);
        a.d[i] = di;
        acc[0] = fma(gi, di, acc[0]);
        acc[1] = fma(di, di, acc[1]);
    }
    if (a.part) block_rows_store<2>(acc, a.part);
}

// xt = x + stp d   (lnsrlb: x = z at stp = 1, else stp d + t)
__global__ void k_trial(double *__restrict__ xt, const double *__restrict__ x, const double *__restrict__ d, double stp,
                        long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        xt[i] = (stp == 1.0) ? x[i] + d[i] : fma(stp, d[i], x[i]);
}

// out[r] = sum over blocks of part[r][.] (one block per row, fixed order)
__global__ void k_finish_rows(const double *__restrict__ part, int nblk, double *__restrict__ out) {
    __shared__ double ss[256];
    const double *row = part + (size_t)blockIdx.x * nblk;
    double s = 0.0;
    for (int i = threadIdx.x; i < nblk; i += blockDim.x) s += row[i];
    ss[threadIdx.x] = s;
    __syncthreads();
    for (int off = blockDim.x / 2; off > 0; off >>= 1) {
        if ((int)threadIdx.x < off) ss[threadIdx.x] += ss[threadIdx.x + off];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = ss[0];
}

}  // namespace mdft
