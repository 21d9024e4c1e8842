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
// Gradient and direction vectors TV: double (FP64 solves) or float (mixed solves); the
// point x (TXP): FP64, or FP32 in the FP32 phase of a mixed solve.  A thread takes V
// consecutive elements per step (16 bytes of TV).
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
    const void *g, *gold, *d;  // vector type TV
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

// V consecutive elements moved as one access (V sizeof(T) bytes, naturally aligned)
template <int B> struct RawT;
template <> struct RawT<2> { using t = unsigned short; };
template <> struct RawT<4> { using t = unsigned int; };
template <> struct RawT<8> { using t = uint2; };
template <> struct RawT<16> { using t = uint4; };
struct alignas(32) Raw32 { uint4 a, b; };
template <> struct RawT<32> { using t = Raw32; };
template <typename T, int V>
__device__ __forceinline__ void vload(const T *p, long long j, T (&v)[V]) {
    using R = typename RawT<V * (int)sizeof(T)>::t;
    const R r = reinterpret_cast<const R *>(p)[j];
    __builtin_memcpy(&v[0], &r, sizeof(R));
}
template <typename T, int V>
__device__ __forceinline__ void vstore(T *p, long long j, const T (&v)[V]) {
    using R = typename RawT<V * (int)sizeof(T)>::t;
    R r;
    __builtin_memcpy(&r, &v[0], sizeof(R));
    reinterpret_cast<R *>(p)[j] = r;
}

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

// V elements per thread and step (V = 1, or 16 bytes of TV when n is a multiple of V)
template <typename TS, typename TV, int K, bool PAIR, bool SELF, int V>
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
    const TV *gp = static_cast<const TV *>(a.g), *gop = static_cast<const TV *>(a.gold), *dp = static_cast<const TV *>(a.d);
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long nv = a.n / V;
    for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < nv; j += stride) {
        TV g[V], go[V], d[V];
        vload<TV, V>(gp, j, g);
        if constexpr (PAIR) vload<TV, V>(gop, j, go);
        if constexpr (PAIR && SELF) vload<TV, V>(dp, j, d);
        TS sc[KK][V], yc[KK][V];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            vload<TS, V>(sv[k], j, sc[k]);
            vload<TS, V>(yv[k], j, yc[k]);
        }
#pragma unroll
        for (int e = 0; e < V; ++e) {
            TS sk[KK], yk[KK];
#pragma unroll
            for (int k = 0; k < K; ++k) {
                sk[k] = sc[k][e];
                yk[k] = yc[k][e];
            }
            pair_dots_elem<TS, K, PAIR, SELF>(a.stp, (double)g[e], PAIR ? (double)go[e] : 0.0, PAIR && SELF ? (double)d[e] : 0.0, acc,
                                              sk, yk);
        }
    }
    block_rows_store<R>(acc, a.part);
}

// d = (accumulate ? d : cg g) + sum_k cv_k v_k.  NEWPAIR (first launch only): the accepted
// pair s_n = stp d_old, y_n = g - gold is formed from the d being replaced, rounded to the
// storage type, stored in snew/ynew and added with coefficients cs_n, cy_n.
struct DirArgs {
    const void *g, *gold;  // vector type TV, as d
    double cg, stp, cs_n, cy_n;
    const void *v[2 * kPairGroup];
    double cv[2 * kPairGroup];
    void *snew, *ynew;
    void *d;
    int accumulate;
    long long n;
    const void *x;  // non-null (last launch): also the first trial point xt = x + stp_t d (type TXP)
    void *xt;
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

template <typename TS, typename TV, typename TXP, int K, bool NEWPAIR, int V>
__global__ void __launch_bounds__(kRedThreads) k_direction(DirArgs a) {
    constexpr int KK = K > 0 ? K : 1;
    const TS *vv[KK];
#pragma unroll
    for (int k = 0; k < K; ++k) vv[k] = static_cast<const TS *>(a.v[k]);
    TS *snew = static_cast<TS *>(a.snew), *ynew = static_cast<TS *>(a.ynew);
    const TV *gp = static_cast<const TV *>(a.g), *gop = static_cast<const TV *>(a.gold);
    TV *dp = static_cast<TV *>(a.d);
    const long long stride = (long long)gridDim.x * blockDim.x;
    const bool need_g = !a.accumulate || NEWPAIR;
    const bool need_d = a.accumulate || NEWPAIR;
    const long long nv = a.n / V;
    for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < nv; j += stride) {
        TV g[V], go[V], d[V];
        if (need_g) vload<TV, V>(gp, j, g);
        if constexpr (NEWPAIR) vload<TV, V>(gop, j, go);
        if (need_d) vload<TV, V>(dp, j, d);
        TS vc[KK][V];
#pragma unroll
        for (int k = 0; k < K; ++k) vload<TS, V>(vv[k], j, vc[k]);
        TV r[V];
        TS sn[V], yn[V];
        double rd[V];
#pragma unroll
        for (int e = 0; e < V; ++e) {
            TS vk[KK];
#pragma unroll
            for (int k = 0; k < K; ++k) vk[k] = vc[k][e];
            sn[e] = (TS)0;
            yn[e] = (TS)0;
            rd[e] = direction_elem<TS, K, NEWPAIR>(a, need_g ? (double)g[e] : 0.0, NEWPAIR ? (double)go[e] : 0.0,
                                                   need_d ? (double)d[e] : 0.0, vk, sn[e], yn[e]);
            r[e] = (TV)rd[e];
        }
        vstore<TV, V>(dp, j, r);
        if (a.x) {
            TXP xv[V], xo[V];
            vload<TXP, V>(static_cast<const TXP *>(a.x), j, xv);
#pragma unroll
            for (int e = 0; e < V; ++e) xo[e] = (TXP)trial_elem((double)xv[e], (double)r[e], a.stp_t);
            vstore<TXP, V>(static_cast<TXP *>(a.xt), j, xo);
        }
        if constexpr (NEWPAIR) {
            vstore<TS, V>(snew, j, sn);
            vstore<TS, V>(ynew, j, yn);
        }
    }
}

// xt = x + stp d   (lnsrlb: x = z at stp = 1, else stp d + t); d of type TV, V per thread
template <typename TV, typename TXP, int V>
__global__ void k_trial(TXP *__restrict__ xt, const TXP *__restrict__ x, const TV *__restrict__ d, double stp, long long n) {
    const long long nv = n / V;
    for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < nv; j += (long long)gridDim.x * blockDim.x) {
        TXP xv[V], xo[V];
        TV dv[V];
        vload<TXP, V>(x, j, xv);
        vload<TV, V>(d, j, dv);
#pragma unroll
        for (int e = 0; e < V; ++e) xo[e] = (TXP)trial_elem((double)xv[e], (double)dv[e], stp);
        vstore<TXP, V>(xt, j, xo);
    }
}

// out = (TO) in, element-wise (precision changes of whole vectors at phase boundaries)
template <typename TI, typename TO>
__global__ void k_convert(TO *__restrict__ out, const TI *__restrict__ in, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = (TO)in[i];
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
