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
// History storage TS: double (FP64 solves, the reference's arithmetic) or float (mixed
// solves: pairs are rounded to FP32 when stored and every product uses the stored values).
// VEC = 2: a thread takes element pairs (n even; all vectors are then 2-element aligned).
// Every reduction is two-stage with the fixed grid kRedBlocks and a fixed summation order
// for a given (grid, VEC), so results are reproducible run to run.
#pragma once

#include "common.cuh"
#include "k_vec.cuh"

namespace mdft {

constexpr int kPairGroup = 8;                 // history slots read per k_pair_dots launch
constexpr int kMaxRows = 4 * kPairGroup + 5;  // reduction rows of one launch

// MODE 0: rows s_i.g [0,K), y_i.g [K,2K), g.g [2K]
// MODE 1: forms s_new = stp d and y_new = g - gold (stored), rows as MODE 0 plus
//         s_i.y_new [2K+1,3K+1), y_i.y_new [3K+1,4K+1), y_new.y_new, y_new.g, s_new.g, s_new.y_new
// MODE 2: y_new read back from ynew; rows as MODE 1 without the last four
struct PairDotsArgs {
    const double *g, *gold, *d;
    const void *s[kPairGroup], *y[kPairGroup];
    void *snew, *ynew;
    double stp;
    long long n;
    double *part;  // [rows][gridDim.x]
};

template <int K, int MODE> __host__ __device__ constexpr int pair_rows() {
    return MODE == 0 ? 2 * K + 1 : (MODE == 1 ? 4 * K + 5 : 4 * K + 1);
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

template <typename TS> struct Pair2;
template <> struct Pair2<double> { using t = double2; };
template <> struct Pair2<float> { using t = float2; };

// one element i: sk, yk are the old slots' values there
template <typename TS, int K, int MODE>
__device__ __forceinline__ void pair_dots_elem(const PairDotsArgs &a, TS *snew, TS *ynew, long long i, double gi, double goldi,
                                               double di, double (&acc)[pair_rows<K, MODE>()], const TS *sk, const TS *yk) {
    double yn = 0.0;
    if constexpr (MODE == 1) {
        const TS ys = (TS)(gi - goldi);
        const TS ss = (TS)((a.stp == 1.0) ? di : a.stp * di);
        snew[i] = ss;
        ynew[i] = ys;
        yn = (double)ys;
        const double sn = (double)ss;
        acc[4 * K + 1] = fma(yn, yn, acc[4 * K + 1]);
        acc[4 * K + 2] = fma(yn, gi, acc[4 * K + 2]);
        acc[4 * K + 3] = fma(sn, gi, acc[4 * K + 3]);
        acc[4 * K + 4] = fma(sn, yn, acc[4 * K + 4]);
    } else if constexpr (MODE == 2) {
        yn = (double)ynew[i];
    }
    acc[2 * K] = fma(gi, gi, acc[2 * K]);
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const double si = (double)sk[k], yi = (double)yk[k];
        acc[k] = fma(si, gi, acc[k]);
        acc[K + k] = fma(yi, gi, acc[K + k]);
        if constexpr (MODE != 0) {
            acc[2 * K + 1 + k] = fma(si, yn, acc[2 * K + 1 + k]);
            acc[3 * K + 1 + k] = fma(yi, yn, acc[3 * K + 1 + k]);
        }
    }
}

template <typename TS, int K, int MODE, int VEC>
__global__ void __launch_bounds__(kRedThreads) k_pair_dots(PairDotsArgs a) {
    constexpr int R = pair_rows<K, MODE>();
    constexpr int KK = K > 0 ? K : 1;
    double acc[R];
#pragma unroll
    for (int r = 0; r < R; ++r) acc[r] = 0.0;
    const TS *sv[KK], *yv[KK];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        sv[k] = static_cast<const TS *>(a.s[k]);
        yv[k] = static_cast<const TS *>(a.y[k]);
    }
    TS *snew = static_cast<TS *>(a.snew), *ynew = static_cast<TS *>(a.ynew);
    const long long stride = (long long)gridDim.x * blockDim.x;
    if constexpr (VEC == 1) {
        for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
            TS sk[KK], yk[KK];
#pragma unroll
            for (int k = 0; k < K; ++k) {
                sk[k] = sv[k][i];
                yk[k] = yv[k][i];
            }
            pair_dots_elem<TS, K, MODE>(a, snew, ynew, i, a.g[i], MODE == 1 ? a.gold[i] : 0.0, MODE == 1 ? a.d[i] : 0.0, acc, sk,
                                        yk);
        }
    } else {
        using P2 = typename Pair2<TS>::t;
        const long long n2 = a.n / 2;
        for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < n2; j += stride) {
            const double2 g2 = reinterpret_cast<const double2 *>(a.g)[j];
            double2 go2 = make_double2(0.0, 0.0), d2 = make_double2(0.0, 0.0);
            if constexpr (MODE == 1) {
                go2 = reinterpret_cast<const double2 *>(a.gold)[j];
                d2 = reinterpret_cast<const double2 *>(a.d)[j];
            }
            TS s0[KK], y0[KK], s1[KK], y1[KK];
#pragma unroll
            for (int k = 0; k < K; ++k) {
                const P2 sp = reinterpret_cast<const P2 *>(sv[k])[j], yp = reinterpret_cast<const P2 *>(yv[k])[j];
                s0[k] = sp.x;
                s1[k] = sp.y;
                y0[k] = yp.x;
                y1[k] = yp.y;
            }
            pair_dots_elem<TS, K, MODE>(a, snew, ynew, 2 * j, g2.x, go2.x, d2.x, acc, s0, y0);
            pair_dots_elem<TS, K, MODE>(a, snew, ynew, 2 * j + 1, g2.y, go2.y, d2.y, acc, s1, y1);
        }
    }
    block_rows_store<R>(acc, a.part);
}

// d = (accumulate ? d : cg g) + sum_k cv_k v_k ; with part: rows g.d, d.d
struct DirArgs {
    const double *g;
    double cg;
    const void *v[2 * kPairGroup];
    double cv[2 * kPairGroup];
    double *d;
    int accumulate;
    long long n;
    double *part;
};

template <typename TS, int K, int VEC>
__global__ void __launch_bounds__(kRedThreads) k_direction(DirArgs a) {
    double acc[2] = {0.0, 0.0};
    const TS *vv[K > 0 ? K : 1];
#pragma unroll
    for (int k = 0; k < K; ++k) vv[k] = static_cast<const TS *>(a.v[k]);
    const long long stride = (long long)gridDim.x * blockDim.x;
    const bool need_g = !a.accumulate || a.part;
    if constexpr (VEC == 1) {
        for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
            const double gi = need_g ? a.g[i] : 0.0;
            double di = a.accumulate ? a.d[i] : a.cg * gi;
#pragma unroll
            for (int k = 0; k < K; ++k) di = fma(a.cv[k], (double)vv[k][i], di);
            a.d[i] = di;
            acc[0] = fma(gi, di, acc[0]);
            acc[1] = fma(di, di, acc[1]);
        }
    } else {
        using P2 = typename Pair2<TS>::t;
        const long long n2 = a.n / 2;
        for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < n2; j += stride) {
            const double2 g2 = need_g ? reinterpret_cast<const double2 *>(a.g)[j] : make_double2(0.0, 0.0);
            double2 d2 = a.accumulate ? reinterpret_cast<const double2 *>(a.d)[j] : make_double2(a.cg * g2.x, a.cg * g2.y);
#pragma unroll
            for (int k = 0; k < K; ++k) {
                const P2 v = reinterpret_cast<const P2 *>(vv[k])[j];
                d2.x = fma(a.cv[k], (double)v.x, d2.x);
                d2.y = fma(a.cv[k], (double)v.y, d2.y);
            }
            reinterpret_cast<double2 *>(a.d)[j] = d2;
            acc[0] = fma(g2.x, d2.x, acc[0]);
            acc[1] = fma(d2.x, d2.x, acc[1]);
            acc[0] = fma(g2.y, d2.y, acc[0]);
            acc[1] = fma(d2.y, d2.y, acc[1]);
        }
    }
    if (a.part) block_rows_store<2>(acc, a.part);
}

// xt = x + stp d   (lnsrlb: x = z at stp = 1, else stp d + t)
__global__ void k_trial(double *__restrict__ xt, const double *__restrict__ x, const double *__restrict__ d, double stp,
                        long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        xt[i] = (stp == 1.0) ? x[i] + d[i] : fma(stp, d[i], x[i]);
}

// the same on element pairs (n even, 16-byte aligned vectors); n2 = n / 2
__global__ void k_trial2(double *__restrict__ xt, const double *__restrict__ x, const double *__restrict__ d, double stp,
                         long long n2) {
    for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < n2; j += (long long)gridDim.x * blockDim.x) {
        const double2 xv = reinterpret_cast<const double2 *>(x)[j], dv = reinterpret_cast<const double2 *>(d)[j];
        double2 r;
        r.x = (stp == 1.0) ? xv.x + dv.x : fma(stp, dv.x, xv.x);
        r.y = (stp == 1.0) ? xv.y + dv.y : fma(stp, dv.y, xv.y);
        reinterpret_cast<double2 *>(xt)[j] = r;
    }
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
