// Angular transforms as per-point dense contractions (FP64 path).
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
#pragma once

#include "common.cuh"

namespace mdft {

constexpr int kAngThreads = 256;
constexpr int kAngBN = 64;  // output columns per chunk
constexpr int kAngBK = 32;  // matrix rows per slab

struct AngularArgs {
    long long N;  // points
    int no, np;
    double rho0;
};

struct GatherArgs {
    long long N;
    int no, np;
    double rho0, kT, dv, prefactor, cst;  // prefactor = -kT 2 (4 pi^2)/mrso/n0, cst = 1/N
    int do_ideal;                         // add F_id, F_ext and their gradient
    int df_mode;                          // 0 none, 1 store (id + exc), 2 accumulate exc
};

// one 32-row slab of the inner product
template <int TM>
__device__ __forceinline__ void ang_slab(const double *__restrict__ As, int lda, const double *__restrict__ Bs, int k0,
                                         int tx, int ty, double (&acc)[TM][4]) {
#pragma unroll 8
    for (int kk = 0; kk < kAngBK; ++kk) {
        const double *ar = As + (size_t)(k0 + kk) * lda + ty * TM;
        double a[TM];
#pragma unroll
        for (int i = 0; i < TM; ++i) a[i] = ar[i];
        const double2 *br = reinterpret_cast<const double2 *>(Bs + kk * kAngBN + tx * 4);
        double2 b01 = br[0], b23 = br[1];
#pragma unroll
        for (int i = 0; i < TM; ++i) {
            acc[i][0] = fma(a[i], b01.x, acc[i][0]);
            acc[i][1] = fma(a[i], b01.y, acc[i][1]);
            acc[i][2] = fma(a[i], b23.x, acc[i][2]);
            acc[i][3] = fma(a[i], b23.y, acc[i][3]);
        }
    }
}

// Load a 32 x 64 slab of the row-major K x J matrix M (zero outside).
__device__ __forceinline__ void ang_load_slab(double *Bs, const double *__restrict__ M, int K, int J, int k0, int j0) {
    for (int f = threadIdx.x; f < kAngBK * kAngBN; f += blockDim.x) {
        int kk = f / kAngBN, jj = f % kAngBN;
        int k = k0 + kk, j = j0 + jj;
        Bs[f] = (k < K && j < J) ? M[(size_t)k * J + j] : 0.0;
    }
}

// S1: xi [N][no] -> planes [np][N] (complex).
template <int BM>
__global__ void __launch_bounds__(kAngThreads) k_project_f64(const double *__restrict__ xi, const double *__restrict__ A,
                                                             double2 *__restrict__ planes, AngularArgs a) {
    constexpr int TM = BM / 16;
    extern __shared__ double smem[];
    const int K = a.no, J = 2 * a.np;
    const int Kpad = (K + kAngBK - 1) / kAngBK * kAngBK;
    const int lda = BM + 1;
    double *As = smem;                          // [Kpad][BM+1]
    double *Bs = As + (size_t)Kpad * lda;       // [BK][BN]
    double2 *Cs = reinterpret_cast<double2 *>(Bs + kAngBK * kAngBN);  // [BN/2][BM]
    const long long pt0 = (long long)blockIdx.x * BM;
    const int npts = (int)min((long long)BM, a.N - pt0);
    // inputs: rho0 (xi^2 - 1), coalesced along io
    for (int f = threadIdx.x; f < BM * Kpad; f += blockDim.x) {
        int p = f / Kpad, k = f % Kpad;
        double v = 0.0;
        if (p < npts && k < K) {
            double x = xi[(pt0 + p) * K + k];
            v = a.rho0 * (x * x - 1.0);
        }
        As[(size_t)k * lda + p] = v;
    }
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    for (int j0 = 0; j0 < J; j0 += kAngBN) {
        double acc[TM][4];
#pragma unroll
        for (int i = 0; i < TM; ++i) acc[i][0] = acc[i][1] = acc[i][2] = acc[i][3] = 0.0;
        for (int k0 = 0; k0 < Kpad; k0 += kAngBK) {
            __syncthreads();
            ang_load_slab(Bs, A, K, J, k0, j0);
            __syncthreads();
            ang_slab<TM>(As, lda, Bs, k0, tx, ty, acc);
        }
        // stage the chunk as complex [ip_local][point]
#pragma unroll
        for (int i = 0; i < TM; ++i) {
            int p = ty * TM + i;
            Cs[(tx * 2 + 0) * BM + p] = make_double2(acc[i][0], acc[i][1]);
            Cs[(tx * 2 + 1) * BM + p] = make_double2(acc[i][2], acc[i][3]);
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

// S7 fused with the ideal + external term.  partial[block] = {F_id, F_ext, sum for F_exc}.
template <int BM>
__global__ void __launch_bounds__(kAngThreads) k_gather_f64(const double2 *__restrict__ planes, const double *__restrict__ B,
                                                            const double *__restrict__ xi, const double *__restrict__ vext,
                                                            const double *__restrict__ w, double *__restrict__ df,
                                                            double *__restrict__ partial, GatherArgs a) {
    constexpr int TM = BM / 16;
    extern __shared__ double smem[];
    const int K = 2 * a.np, J = a.no;
    const int Kpad = (K + kAngBK - 1) / kAngBK * kAngBK;
    const int lda = BM + 1;
    double *As = smem;                     // [Kpad][BM+1]
    double *Bs = As + (size_t)Kpad * lda;  // [BK][BN]
    double *Cs = Bs + kAngBK * kAngBN;     // [BM][BN+1]
    __shared__ double red[3][kAngThreads / 32];
    const long long pt0 = (long long)blockIdx.x * BM;
    const int npts = (int)min((long long)BM, a.N - pt0);
    for (int f = threadIdx.x; f < (Kpad / 2) * BM; f += blockDim.x) {
        int ip = f / BM, p = f % BM;
        double2 v = make_double2(0.0, 0.0);
        if (p < npts && ip < a.np) {
            v = planes[(size_t)ip * a.N + pt0 + p];
            v.x *= a.cst;
            v.y *= a.cst;
        }
        As[(size_t)(2 * ip) * lda + p] = v.x;
        As[(size_t)(2 * ip + 1) * lda + p] = v.y;
    }
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    double fid = 0.0, fext = 0.0, fexc = 0.0;
    for (int j0 = 0; j0 < J; j0 += kAngBN) {
        double acc[TM][4];
#pragma unroll
        for (int i = 0; i < TM; ++i) acc[i][0] = acc[i][1] = acc[i][2] = acc[i][3] = 0.0;
        for (int k0 = 0; k0 < Kpad; k0 += kAngBK) {
            __syncthreads();
            ang_load_slab(Bs, B, K, J, k0, j0);
            __syncthreads();
            ang_slab<TM>(As, lda, Bs, k0, tx, ty, acc);
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
            double vexc = a.prefactor * wio * Cs[p * (kAngBN + 1) + jj];
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
            if (a.df_mode == 1) df[g] = did + dexc;
            else if (a.df_mode == 2) df[g] = df[g] + dexc;
        }
    }
    // block reduction (fixed order -> deterministic)
    for (int off = 16; off > 0; off >>= 1) {
        fid += __shfl_down_sync(0xffffffffu, fid, off);
        fext += __shfl_down_sync(0xffffffffu, fext, off);
        fexc += __shfl_down_sync(0xffffffffu, fexc, off);
    }
    int wid = threadIdx.x / 32, lane = threadIdx.x % 32;
    if (lane == 0) {
        red[0][wid] = fid;
        red[1][wid] = fext;
        red[2][wid] = fexc;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s0 = 0, s1 = 0, s2 = 0;
        for (int i = 0; i < kAngThreads / 32; ++i) {
            s0 += red[0][i];
            s1 += red[1][i];
            s2 += red[2][i];
        }
        partial[3 * (size_t)blockIdx.x + 0] = s0;
        partial[3 * (size_t)blockIdx.x + 1] = s1;
        partial[3 * (size_t)blockIdx.x + 2] = s2;
    }
}

inline size_t project_smem_bytes(int BM, int no) {
    int Kpad = (no + kAngBK - 1) / kAngBK * kAngBK;
    return sizeof(double) * ((size_t)Kpad * (BM + 1) + kAngBK * kAngBN) + sizeof(double2) * (kAngBN / 2) * BM;
}
inline size_t gather_smem_bytes(int BM, int np) {
    int Kpad = (2 * np + kAngBK - 1) / kAngBK * kAngBK;
    return sizeof(double) * ((size_t)Kpad * (BM + 1) + kAngBK * kAngBN + (size_t)BM * (kAngBN + 1));
}

// Sum n rows of 3 partials into out[3] (one block, fixed order).
__global__ void k_reduce3(const double *__restrict__ partial, long long n, double *__restrict__ out) {
    __shared__ double s[3][256];
    double a0 = 0, a1 = 0, a2 = 0;
    for (long long i = threadIdx.x; i < n; i += blockDim.x) {
        a0 += partial[3 * i + 0];
        a1 += partial[3 * i + 1];
        a2 += partial[3 * i + 2];
    }
    s[0][threadIdx.x] = a0;
    s[1][threadIdx.x] = a1;
    s[2][threadIdx.x] = a2;
    __syncthreads();
    for (int off = blockDim.x / 2; off > 0; off >>= 1) {
        if ((int)threadIdx.x < off) {
            s[0][threadIdx.x] += s[0][threadIdx.x + off];
            s[1][threadIdx.x] += s[1][threadIdx.x + off];
            s[2][threadIdx.x] += s[2][threadIdx.x + off];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = s[0][0];
        out[1] = s[1][0];
        out[2] = s[2][0];
    }
}

}  // namespace mdft
