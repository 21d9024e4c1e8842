// Angular transforms as per-point dense contractions, templated on the compute
// precision T (double: parity path; float: mixed path).
//
//  project (S1, src/module_energy_cproj_mrso.f90:276-290 with angl2proj):
//     drho_p[ip][r] = sum_io rho0 (xi[r][io]^2 - 1) A[io][ip]
//  gather (S7, src/module_energy_cproj_mrso.f90:728-762 with proj2angl), fused
//  with the ideal and external terms (src/module_energy_ideal_and_external.f90:46-73):
//     vexc[r][io] = P w(io) sum_ip gamma_p[ip][r]/N . B[ip][io]
//
// Both are [points x K] . [K x J] products with K, J <= a few hundred: a CTA
// stages BM points x K inputs in shared memory (coalesced: a point's no
// doubles are contiguous, a projection plane's points are contiguous), the
// matrix in 32-row slabs, and each thread keeps a (BM/16) x 4 register tile.
// xi, vext, df, the epilogue arithmetic (log, ideal and external terms) and all
// partial sums are FP64 in both precisions.
#pragma once

#include "common.cuh"
#include "k_fft.cuh"

namespace mdft {

constexpr int kAngThreads = 256;
constexpr int kAngBN = 64;  // output columns per chunk
constexpr int kAngBK = 32;  // matrix rows per slab

struct AngularArgs {
    long long N;  // points
    int no, np;
    double rho0;
};

// per-block partials of the gathers: F_id, F_ext, F_exc sum, df.d, max|df|, sum w df
constexpr int kGatherSums = 6;

struct GatherArgs {
    long long N;
    int no, np;
    double rho0, kT, dv, prefactor, cst;  // prefactor = -kT 2 (4 pi^2)/mrso/n0, cst = 1/N
    int do_ideal;                         // add F_id, F_ext and their gradient
    int df_mode;                          // 0 none, 1 store (id + exc), 2 accumulate exc
    const void *dvec;                     // df_mode 1: also df.dvec (null: df.df is not wanted -> 0);
                                          // FP64, or the type of df in k_gather_tma
    int fail_wait;                        // the bulk-copy gathers report a timed-out wait at once,
                                          // before any copy or tensor-memory allocation (tests)
};

template <typename T> struct Vec4;
template <> struct Vec4<double> { struct t { double2 a, b; }; };
template <> struct Vec4<float> { using t = float4; };
__device__ __forceinline__ void unpack4(const Vec4<double>::t &v, double (&o)[4]) { o[0] = v.a.x; o[1] = v.a.y; o[2] = v.b.x; o[3] = v.b.y; }
__device__ __forceinline__ void unpack4(const float4 &v, float (&o)[4]) { o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w; }

// one 32-row slab of the inner product
template <typename T, int TM>
__device__ __forceinline__ void ang_slab(const T *__restrict__ As, int lda, const T *__restrict__ Bs, int k0, int tx, int ty,
                                         T (&acc)[TM][4]) {
#pragma unroll 8
    for (int kk = 0; kk < kAngBK; ++kk) {
        const T *ar = As + (size_t)(k0 + kk) * lda + ty * TM;
        T a[TM];
#pragma unroll
        for (int i = 0; i < TM; ++i) a[i] = ar[i];
        T b[4];
        unpack4(*reinterpret_cast<const typename Vec4<T>::t *>(Bs + kk * kAngBN + tx * 4), b);
#pragma unroll
        for (int i = 0; i < TM; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
}

// Load a 32 x 64 slab of the row-major K x J matrix M (zero outside).
template <typename T>
__device__ __forceinline__ void ang_load_slab(T *Bs, const T *__restrict__ M, int K, int J, int k0, int j0) {
    for (int f = threadIdx.x; f < kAngBK * kAngBN; f += blockDim.x) {
        int kk = f / kAngBN, jj = f % kAngBN;
        int k = k0 + kk, j = j0 + jj;
        Bs[f] = (k < K && j < J) ? M[(size_t)k * J + j] : (T)0;
    }
}

// S1: xi [N][no] (FP64) -> planes [np][N] (complex T).
template <typename T, int BM>
__global__ void __launch_bounds__(kAngThreads) k_project(const double *__restrict__ xi, const T *__restrict__ A,
                                                         typename Cplx<T>::t *__restrict__ planes, AngularArgs a) {
    using C = typename Cplx<T>::t;
    constexpr int TM = BM / 16;
    extern __shared__ __align__(16) unsigned char ang_smem[];
    T *smem = reinterpret_cast<T *>(ang_smem);
    const int K = a.no, J = 2 * a.np;
    const int Kpad = (K + kAngBK - 1) / kAngBK * kAngBK;
    const int lda = BM + 1;
    T *As = smem;                                                   // [Kpad][BM+1]
    T *Bs = As + ((size_t)Kpad * lda + 3) / 4 * 4;                  // [BK][BN], 16-byte aligned
    C *Cs = reinterpret_cast<C *>(Bs + kAngBK * kAngBN);            // [BN/2][BM]
    const long long pt0 = (long long)blockIdx.x * BM;
    const int npts = (int)min((long long)BM, a.N - pt0);
    for (int f = threadIdx.x; f < BM * Kpad; f += blockDim.x) {
        int p = f / Kpad, k = f % Kpad;
        T v = 0;
        if (p < npts && k < K) {
            double x = xi[(pt0 + p) * K + k];
            v = (T)(a.rho0 * (x * x - 1.0));
        }
        As[(size_t)k * lda + p] = v;
    }
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    for (int j0 = 0; j0 < J; j0 += kAngBN) {
        T acc[TM][4];
#pragma unroll
        for (int i = 0; i < TM; ++i) acc[i][0] = acc[i][1] = acc[i][2] = acc[i][3] = (T)0;
        for (int k0 = 0; k0 < Kpad; k0 += kAngBK) {
            __syncthreads();
            ang_load_slab<T>(Bs, A, K, J, k0, j0);
            __syncthreads();
            ang_slab<T, TM>(As, lda, Bs, k0, tx, ty, acc);
        }
#pragma unroll
        for (int i = 0; i < TM; ++i) {
            int p = ty * TM + i;
            C u, v;
            u.x = acc[i][0]; u.y = acc[i][1];
            v.x = acc[i][2]; v.y = acc[i][3];
            Cs[(tx * 2 + 0) * BM + p] = u;
            Cs[(tx * 2 + 1) * BM + p] = v;
        }
        __syncthreads();
        const int ip0 = j0 / 2;
        for (int f = threadIdx.x; f < (kAngBN / 2) * BM; f += blockDim.x) {
            int il = f / BM, p = f % BM;
            int ip = ip0 + il;
            if (ip < a.np && p < npts) planes[(size_t)ip * a.N + pt0 + p] = Cs[il * BM + p];
        }
    }
}

// S7 fused with the ideal + external term.  partial[block] = {F_id, F_ext, sum for F_exc,
// df.dvec, max|df|} (the last two only with df_mode 1: the line-search slope and the
// projected-gradient norm of the minimiser come out of the same pass).
template <typename T, int BM>
__global__ void __launch_bounds__(kAngThreads) k_gather(const typename Cplx<T>::t *__restrict__ planes, const T *__restrict__ B,
                                                        const double *__restrict__ xi, const double *__restrict__ vext,
                                                        const double *__restrict__ w, double *__restrict__ df,
                                                        double *__restrict__ partial, GatherArgs a) {
    using C = typename Cplx<T>::t;
    constexpr int TM = BM / 16;
    extern __shared__ __align__(16) unsigned char ang_smem[];
    T *smem = reinterpret_cast<T *>(ang_smem);
    const int K = 2 * a.np, J = a.no;
    const int Kpad = (K + kAngBK - 1) / kAngBK * kAngBK;
    const int lda = BM + 1;
    T *As = smem;                                    // [Kpad][BM+1]
    T *Bs = As + ((size_t)Kpad * lda + 3) / 4 * 4;   // [BK][BN]
    T *Cs = Bs + kAngBK * kAngBN;                    // [BM][BN+1]
    __shared__ double red[kGatherSums][kAngThreads / 32];
    const long long pt0 = (long long)blockIdx.x * BM;
    const int npts = (int)min((long long)BM, a.N - pt0);
    const T cst = (T)a.cst;
    for (int f = threadIdx.x; f < (Kpad / 2) * BM; f += blockDim.x) {
        int ip = f / BM, p = f % BM;
        C v;
        v.x = 0;
        v.y = 0;
        if (p < npts && ip < a.np) {
            v = planes[(size_t)ip * a.N + pt0 + p];
            v.x *= cst;
            v.y *= cst;
        }
        As[(size_t)(2 * ip) * lda + p] = v.x;
        As[(size_t)(2 * ip + 1) * lda + p] = v.y;
    }
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    double fid = 0.0, fext = 0.0, fexc = 0.0, gdv = 0.0, gmx = 0.0, gun = 0.0;
    for (int j0 = 0; j0 < J; j0 += kAngBN) {
        T acc[TM][4];
#pragma unroll
        for (int i = 0; i < TM; ++i) acc[i][0] = acc[i][1] = acc[i][2] = acc[i][3] = (T)0;
        for (int k0 = 0; k0 < Kpad; k0 += kAngBK) {
            __syncthreads();
            ang_load_slab<T>(Bs, B, K, J, k0, j0);
            __syncthreads();
            ang_slab<T, TM>(As, lda, Bs, k0, tx, ty, acc);
        }
#pragma unroll
        for (int i = 0; i < TM; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) Cs[(ty * TM + i) * (kAngBN + 1) + tx * 4 + j] = acc[i][j];
        __syncthreads();
        for (int f = threadIdx.x; f < BM * kAngBN; f += blockDim.x) {
            int p = f / kAngBN, jj = f % kAngBN, io = j0 + jj;
            if (p >= npts || io >= J) continue;
            size_t g = (size_t)(pt0 + p) * J + io;
            double wio = w[io];
            double vexc = a.prefactor * wio * (double)Cs[p * (kAngBN + 1) + jj];
            double x = xi[g];
            fexc += (x * x * a.rho0 - a.rho0) * vexc;
            double dexc = 2.0 * a.rho0 * x * vexc;
            double did = 0.0;
            if (a.do_ideal) {
                double v = vext[g];
                double rho = x * x * a.rho0;
                if (rho > kEpsDp) {
                    double lg = log(rho / a.rho0);
                    fid += a.kT * a.dv * wio * (rho * lg - rho + a.rho0);
                    fext += a.dv * wio * rho * v;
                    did = wio * 2.0 * a.rho0 * x * (a.kT * lg + v);
                } else {
                    fid += a.kT * a.dv * wio * a.rho0;
                }
            }
            if (a.df_mode == 1) {
                const double gv = did + dexc;
                df[g] = gv;
                if (a.dvec) gdv = fma(gv, static_cast<const double *>(a.dvec)[g], gdv);
                gmx = fmax(gmx, fabs(gv));
                gun = fma(gv, wio, gun);
            } else if (a.df_mode == 2) {
                df[g] = df[g] + dexc;
            }
        }
    }
    // block reduction (fixed order -> deterministic)
    for (int off = 16; off > 0; off >>= 1) {
        fid += __shfl_down_sync(0xffffffffu, fid, off);
        fext += __shfl_down_sync(0xffffffffu, fext, off);
        fexc += __shfl_down_sync(0xffffffffu, fexc, off);
        gdv += __shfl_down_sync(0xffffffffu, gdv, off);
        gmx = fmax(gmx, __shfl_down_sync(0xffffffffu, gmx, off));
        gun += __shfl_down_sync(0xffffffffu, gun, off);
    }
    int wid = threadIdx.x / 32, lane = threadIdx.x % 32;
    if (lane == 0) {
        red[0][wid] = fid;
        red[1][wid] = fext;
        red[2][wid] = fexc;
        red[3][wid] = gdv;
        red[4][wid] = gmx;
        red[5][wid] = gun;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s0 = 0, s1 = 0, s2 = 0, s3 = 0, s4 = 0, s5 = 0;
        for (int i = 0; i < kAngThreads / 32; ++i) {
            s0 += red[0][i];
            s1 += red[1][i];
            s2 += red[2][i];
            s3 += red[3][i];
            s4 = fmax(s4, red[4][i]);
            s5 += red[5][i];
        }
        double *pp = partial + kGatherSums * (size_t)blockIdx.x;
        pp[0] = s0;
        pp[1] = s1;
        pp[2] = s2;
        pp[3] = s3;
        pp[4] = s4;
        pp[5] = s5;
    }
}

template <typename T>
inline size_t project_smem_bytes(int BM, int no) {
    int Kpad = (no + kAngBK - 1) / kAngBK * kAngBK;
    return sizeof(T) * (((size_t)Kpad * (BM + 1) + 3) / 4 * 4 + kAngBK * kAngBN) + sizeof(typename Cplx<T>::t) * (kAngBN / 2) * BM;
}
template <typename T>
inline size_t gather_smem_bytes(int BM, int np) {
    int Kpad = (2 * np + kAngBK - 1) / kAngBK * kAngBK;
    return sizeof(T) * (((size_t)Kpad * (BM + 1) + 3) / 4 * 4 + kAngBK * kAngBN + (size_t)BM * (kAngBN + 1));
}

// Sum n rows of kGatherSums partials into out[0..5] (one block, fixed order): entry 4 is a
// maximum, the others sums.
__global__ void k_reduce_sums(const double *__restrict__ partial, long long n, double *__restrict__ out) {
    __shared__ double s[kGatherSums][256];
    double a[kGatherSums] = {0, 0, 0, 0, 0, 0};
    for (long long i = threadIdx.x; i < n; i += blockDim.x) {
        const double *pp = partial + kGatherSums * i;
        for (int j = 0; j < kGatherSums; ++j) a[j] = j == 4 ? fmax(a[j], pp[j]) : a[j] + pp[j];
    }
    for (int j = 0; j < kGatherSums; ++j) s[j][threadIdx.x] = a[j];
    __syncthreads();
    for (int off = blockDim.x / 2; off > 0; off >>= 1) {
        if ((int)threadIdx.x < off) {
            for (int j = 0; j < kGatherSums; ++j)
                s[j][threadIdx.x] = j == 4 ? fmax(s[j][threadIdx.x], s[j][threadIdx.x + off]) : s[j][threadIdx.x] + s[j][threadIdx.x + off];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int j = 0; j < kGatherSums; ++j) out[j] = s[j][0];
}

}  // namespace mdft
