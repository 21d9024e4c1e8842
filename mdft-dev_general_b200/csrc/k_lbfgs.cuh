// Vector passes of the limited-memory BFGS driver in compact form.
//
// The search direction -H g of src/module_lbfgs_nocedal_mdft.f90 (formk/cmprlb/subsm with
// no bounds) is formed as  d = cg g + sum_i a_i s_i + sum_i b_i y_i  with the 2m+1
// coefficients computed on the host from small Gram matrices (Byrd, Nocedal and Schnabel,
// Math. Prog. 63 (1994), eq. 3.1 in inverse form).  A step therefore reads each history
// vector twice -- once for its inner products with the trial gradient (k_pair_dots, run
// right after each trial evaluation, before the one host synchronisation of the step), once
// for the combination (k_direction, which also stores the accepted pair) -- instead of the
// four passes per pair of the two-loop recursion.
//
// History storage TS: double (FP64 solves, the reference's arithmetic) or __nv_bfloat16
// (mixed solves: pairs are rounded to BF16 when stored and every product, in FP64, uses the
// stored values, so the compact matrix stays the exact BFGS matrix of the stored pairs).
// VEC = 2: a thread takes element pairs (n even; all vectors are then 2-element aligned).
// Every reduction is two-stage with the fixed grid kRedBlocks and a fixed summation order
// for a given (grid, VEC), so results are reproducible run to run.
#pragma once

#include "common.cuh"
#include "k_vec.cuh"

#include <cuda_bf16.h>

namespace mdft {

constexpr int kPairGroup = 8;                 // history slots read per k_pair_dots launch
constexpr int kMaxRows = 4 * kPairGroup + 5;  // reduction rows of one k_pair_dots launch

// Inner products of the history slots s_i, y_i (K of them) with a gradient g:
//   rows s_i.g [0,K), y_i.g [K,2K), g.g [2K]
// PAIR: also with the candidate pair s_n = stp d, y_n = g - gold, formed on the fly and
//   rounded to the storage type exactly as k_direction will store it (nothing is written):
//   rows s_i.y_n [2K+1,3K+1), y_i.y_n [3K+1,4K+1)
// SELF (with PAIR): the candidate's own rows y_n.y_n, y_n.g, s_n.g, s_n.y_n [4K+1,4K+5)
struct PairDotsArgs {
    const double *g, *gold, *d;
    const void *s[kPairGroup], *y[kPairGroup];
    double stp;
    long long n;
    double *part;  // [rows][gridDim.x]
};

__host__ __device__ constexpr int pair_rows(int K, bool pair, bool self) {
    return 2 * K + 1 + (pair ? 2 * K : 0) + (pair && self ? 4 : 0);
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
template <> struct Pair2<__nv_bfloat16> { using t = __nv_bfloat162; };

// one element: sk, yk are the slots' values there
template <typename TS, int K, bool PAIR, bool SELF>
__device__ __forceinline__ void pair_dots_elem(double stp, double gi, double goldi, double di, double (&acc)[pair_rows(K, PAIR, SELF)],
                                               const TS *sk, const TS *yk) {
    double yn = 0.0;
    if constexpr (PAIR) {
        yn = (double)(TS)(gi - goldi);
        if constexpr (SELF) {
            const double sn = (double)(TS)((stp == 1.0) ? di : stp * di);
            acc[4 * K + 1] = fma(yn, yn, acc[4 * K + 1]);
            acc[4 * K + 2] = fma(yn, gi, acc[4 * K + 2]);
            acc[4 * K + 3] = fma(sn, gi, acc[4 * K + 3]);
            acc[4 * K + 4] = fma(sn, yn, acc[4 * K + 4]);
        }
    }
    acc[2 * K] = fma(gi, gi, acc[2 * K]);
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const double si = (double)sk[k], yi = (double)yk[k];
        acc[k] = fma(si, gi, acc[k]);
        acc[K + k] = fma(yi, gi, acc[K + k]);
        if constexpr (PAIR) {
            acc[2 * K + 1 + k] = fma(si, yn, acc[2 * K + 1 + k]);
            acc[3 * K + 1 + k] = fma(yi, yn, acc[3 * K + 1 + k]);
        }
    }
}

template <typename TS, int K, bool PAIR, bool SELF, int VEC>
__global__ void __launch_bounds__(kRedThreads) k_pair_dots(PairDotsArgs a) {
    constexpr int R = pair_rows(K, PAIR, SELF);
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
    const long long stride = (long long)gridDim.x * blockDim.x;
    if constexpr (VEC == 1) {
        for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
            TS sk[KK], yk[KK];
#pragma unroll
            for (int k = 0; k < K; ++k) {
                sk[k] = sv[k][i];
                yk[k] = yv[k][i];
            }
            pair_dots_elem<TS, K, PAIR, SELF>(a.stp, a.g[i], PAIR ? a.gold[i] : 0.0, PAIR && SELF ? a.d[i] : 0.0, acc, sk, yk);
        }
    } else {
        using P2 = typename Pair2<TS>::t;
        const long long n2 = a.n / 2;
        for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < n2; j += stride) {
            const double2 g2 = reinterpret_cast<const double2 *>(a.g)[j];
            double2 go2 = make_double2(0.0, 0.0), d2 = make_double2(0.0, 0.0);
            if constexpr (PAIR) go2 = reinterpret_cast<const double2 *>(a.gold)[j];
            if constexpr (PAIR && SELF) d2 = reinterpret_cast<const double2 *>(a.d)[j];
            TS s0[KK], y0[KK], s1[KK], y1[KK];
#pragma unroll
            for (int k = 0; k < K; ++k) {
                const P2 sp = reinterpret_cast<const P2 *>(sv[k])[j], yp = reinterpret_cast<const P2 *>(yv[k])[j];
                s0[k] = sp.x;
                s1[k] = sp.y;
                y0[k] = yp.x;
                y1[k] = yp.y;
            }
            pair_dots_elem<TS, K, PAIR, SELF>(a.stp, g2.x, go2.x, d2.x, acc, s0, y0);
            pair_dots_elem<TS, K, PAIR, SELF>(a.stp, g2.y, go2.y, d2.y, acc, s1, y1);
        }
    }
    block_rows_store<R>(acc, a.part);
}

// d = (accumulate ? d : cg g) + sum_k cv_k v_k.  NEWPAIR (first launch only): the accepted
// pair s_n = stp d_old, y_n = g - gold is formed from the d being replaced, rounded to the
// storage type, stored in snew/ynew and added with coefficients cs_n, cy_n.
struct DirArgs {
    const double *g, *gold;
    double cg, stp, cs_n, cy_n;
    const void *v[2 * kPairGroup];
    double cv[2 * kPairGroup];
    void *snew, *ynew;
    double *d;
    int accumulate;
    long long n;
    const double *x;  // non-null (last launch): also the first trial point xt = x + stp_t d
    double *xt;
    double stp_t;
};

// the trial point of lnsrlb: x = z at stp = 1, else stp d + t
__device__ __forceinline__ double trial_elem(double x, double d, double stp) { return (stp == 1.0) ? x + d : fma(stp, d, x); }

template <typename TS, int K, bool NEWPAIR>
__device__ __forceinline__ double direction_elem(const DirArgs &a, double gi, double goldi, double dold, const TS *vk, TS &sn,
                                                 TS &yn) {
    double di = a.accumulate ? dold : a.cg * gi;
    if constexpr (NEWPAIR) {
        sn = (TS)((a.stp == 1.0) ? dold : a.stp * dold);
        yn = (TS)(gi - goldi);
        di = fma(a.cs_n, (double)sn, di);
        di = fma(a.cy_n, (double)yn, di);
    }
#pragma unroll
    for (int k = 0; k < K; ++k) di = fma(a.cv[k], (double)vk[k], di);
    return di;
}

template <typename TS, int K, bool NEWPAIR, int VEC>
__global__ void __launch_bounds__(kRedThreads) k_direction(DirArgs a) {
    constexpr int KK = K > 0 ? K : 1;
    const TS *vv[KK];
#pragma unroll
    for (int k = 0; k < K; ++k) vv[k] = static_cast<const TS *>(a.v[k]);
    TS *snew = static_cast<TS *>(a.snew), *ynew = static_cast<TS *>(a.ynew);
    const long long stride = (long long)gridDim.x * blockDim.x;
    const bool need_g = !a.accumulate || NEWPAIR;
    const bool need_d = a.accumulate || NEWPAIR;
    if constexpr (VEC == 1) {
        for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
            TS vk[KK], sn = 0, yn = 0;
#pragma unroll
            for (int k = 0; k < K; ++k) vk[k] = vv[k][i];
            const double di = direction_elem<TS, K, NEWPAIR>(a, need_g ? a.g[i] : 0.0, NEWPAIR ? a.gold[i] : 0.0,
                                                            need_d ? a.d[i] : 0.0, vk, sn, yn);
            a.d[i] = di;
            if (a.x) a.xt[i] = trial_elem(a.x[i], di, a.stp_t);
            if constexpr (NEWPAIR) {
                snew[i] = sn;
                ynew[i] = yn;
            }
        }
    } else {
        using P2 = typename Pair2<TS>::t;
        const long long n2 = a.n / 2;
        for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < n2; j += stride) {
            const double2 g2 = need_g ? reinterpret_cast<const double2 *>(a.g)[j] : make_double2(0.0, 0.0);
            const double2 go2 = NEWPAIR ? reinterpret_cast<const double2 *>(a.gold)[j] : make_double2(0.0, 0.0);
            const double2 d2 = need_d ? reinterpret_cast<const double2 *>(a.d)[j] : make_double2(0.0, 0.0);
            TS v0[KK], v1[KK];
#pragma unroll
            for (int k = 0; k < K; ++k) {
                const P2 v = reinterpret_cast<const P2 *>(vv[k])[j];
                v0[k] = v.x;
                v1[k] = v.y;
            }
            TS s0 = 0, y0 = 0, s1 = 0, y1 = 0;
            double2 r;
            r.x = direction_elem<TS, K, NEWPAIR>(a, g2.x, go2.x, d2.x, v0, s0, y0);
            r.y = direction_elem<TS, K, NEWPAIR>(a, g2.y, go2.y, d2.y, v1, s1, y1);
            reinterpret_cast<double2 *>(a.d)[j] = r;
            if (a.x) {
                const double2 xv = reinterpret_cast<const double2 *>(a.x)[j];
                reinterpret_cast<double2 *>(a.xt)[j] = make_double2(trial_elem(xv.x, r.x, a.stp_t), trial_elem(xv.y, r.y, a.stp_t));
            }
            if constexpr (NEWPAIR) {
                P2 sp, yp;
                sp.x = s0;
                sp.y = s1;
                yp.x = y0;
                yp.y = y1;
                reinterpret_cast<P2 *>(snew)[j] = sp;
                reinterpret_cast<P2 *>(ynew)[j] = yp;
            }
        }
    }
}

// xt = x + stp d   (lnsrlb: x = z at stp = 1, else stp d + t)
__global__ void k_trial(double *__restrict__ xt, const double *__restrict__ x, const double *__restrict__ d, double stp,
                        long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        xt[i] = trial_elem(x[i], d[i], stp);
}

// the same on element pairs (n even, 16-byte aligned vectors); n2 = n / 2
__global__ void k_trial2(double *__restrict__ xt, const double *__restrict__ x, const double *__restrict__ d, double stp,
                         long long n2) {
    for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < n2; j += (long long)gridDim.x * blockDim.x) {
        const double2 xv = reinterpret_cast<const double2 *>(x)[j], dv = reinterpret_cast<const double2 *>(d)[j];
        double2 r;
        r.x = trial_elem(xv.x, dv.x, stp);
        r.y = trial_elem(xv.y, dv.y, stp);
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
