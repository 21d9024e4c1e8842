// S1 projection (angl2proj, src/module_energy_cproj_mrso.f90:276-290; same arithmetic as
// k_project) as a persistent pipeline: one CTA per SM walks the 64-point tiles blockIdx.x,
// +gridDim.x, ...  Thread 0 issues one bulk copy of the tile's xi (64 x no FP64,
// contiguous) into one of two shared-memory stages, so the next tile is in flight while the
// current one is computed.  Each tile is converted once into drho = rho0 (xi^2 - 1) in the
// working precision, transposed to [io][point] so that a lane reads its own point's values
// without bank conflicts.  The matrix A (no x 2np) stays in shared memory for the launch.
//
// Warp w owns projections 4w..4w+3 (8 real columns, read as two broadcast vector loads per
// io) and lane l the points l and l+32, so each plane store is a coalesced 256- or 512-byte
// run.  Used when N is a multiple of 64, np <= 32 (mmax <= 3), xi is 16-byte aligned and
// the stages fit; k_project covers the rest.
#pragma once

#include "common.cuh"
#include "k_angular.cuh"
#include "k_fft.cuh"
#include "k_tma.cuh"

namespace mdft {

constexpr int kPtBM = 64;      // points per tile
constexpr int kPtStages = 2;
constexpr int kPtLd = kPtBM + 1;  // padded row of the transposed tile

inline int pt_warps(int np) { return (np + 3) / 4; }
template <typename T, typename TX = double>
inline size_t project_tma_smem_bytes(int np, int no) {
    const size_t a = (size_t)no * 8 * pt_warps(np) * sizeof(T);
    const size_t dr = ((size_t)no * kPtLd * sizeof(T) + 15) / 16 * 16;
    const size_t st = (size_t)kPtBM * no * sizeof(TX);
    return (a + 15) / 16 * 16 + dr + kPtStages * st;
}

template <typename T> struct Vec8;
template <> struct Vec8<float> {
    static __device__ __forceinline__ void load(const float *p, float (&v)[8]) {
        const float4 x = reinterpret_cast<const float4 *>(p)[0], y = reinterpret_cast<const float4 *>(p)[1];
        v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w; v[4] = y.x; v[5] = y.y; v[6] = y.z; v[7] = y.w;
    }
};
template <> struct Vec8<double> {
    static __device__ __forceinline__ void load(const double *p, double (&v)[8]) {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const double2 x = reinterpret_cast<const double2 *>(p)[k];
            v[2 * k] = x.x;
            v[2 * k + 1] = x.y;
        }
    }
};

// TX: type of xi (double, or float in the FP32 phase of a mixed solve)
template <typename T, typename TX = double>
__global__ void __launch_bounds__(256, sizeof(TX) == 4 ? 2 : 1) k_project_tma(const TX *__restrict__ xi, const T *__restrict__ A,
                                                        typename Cplx<T>::t *__restrict__ planes, int *__restrict__ err,
                                                        AngularArgs a, int ntiles) {
    using C = typename Cplx<T>::t;
    const int no = a.no, np = a.np;
    const int nw = (np + 3) / 4, NC = 8 * nw;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    extern __shared__ __align__(128) unsigned char pt_smem[];
    T *As = reinterpret_cast<T *>(pt_smem);  // [no][NC]
    T *dr = reinterpret_cast<T *>(pt_smem + ((size_t)no * NC * sizeof(T) + 15) / 16 * 16);  // [no][kPtLd]
    unsigned char *stage0 = reinterpret_cast<unsigned char *>(dr) + ((size_t)no * kPtLd * sizeof(T) + 15) / 16 * 16;
    const size_t sbytes = (size_t)kPtBM * no * sizeof(TX);
    __shared__ uint64_t full[kPtStages];
    __shared__ int abort_flag;
    const int nmine = (int)blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;

    auto issue = [&](int i) {  // thread 0
        const int s = i % kPtStages;
        const long long pt0 = (long long)((int)blockIdx.x + i * (int)gridDim.x) * kPtBM;
        mbar_arrive_expect_tx(&full[s], (uint32_t)sbytes);
        bulk_load(stage0 + s * sbytes, xi + pt0 * no, (uint32_t)sbytes, &full[s]);
    };
    if (tid == 0) {
        for (int s = 0; s < kPtStages; ++s) mbar_init(&full[s], 1);
        mbar_fence_init();
        abort_flag = 0;
        for (int i = 0; i < kPtStages && i < nmine; ++i) issue(i);
    }
    for (int f = tid; f < no * NC; f += blockDim.x) {
        const int io = f / NC, j = f % NC;
        As[f] = j < 2 * np ? A[(size_t)io * 2 * np + j] : (T)0;
    }
    __syncthreads();

    for (int i = 0; i < nmine; ++i) {
        const int s = i % kPtStages;
        const bool ok = mbar_wait(&full[s], (uint32_t)((i / kPtStages) & 1));
        if (!ok) abort_flag = 1;
        if (ok) {
            const TX *xs = reinterpret_cast<const TX *>(stage0 + s * sbytes);
            for (int e = tid; e < kPtBM * no; e += blockDim.x) {
                const int p = e / no, io = e % no;
                const double x = (double)xs[e];
                dr[io * kPtLd + p] = (T)(a.rho0 * (x * x - 1.0));
            }
        }
        __syncthreads();  // transposed tile ready, stage s consumed
        if (abort_flag) break;
        if (tid == 0 && i + kPtStages < nmine) issue(i + kPtStages);
        if (warp < nw) {
            T acc[2][8];
#pragma unroll
            for (int p = 0; p < 2; ++p)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[p][j] = (T)0;
            const T *ar = As + 8 * warp;
#pragma unroll 4
            for (int io = 0; io < no; ++io) {
                const T d0 = dr[io * kPtLd + lane], d1 = dr[io * kPtLd + lane + 32];
                T b[8];
                Vec8<T>::load(ar + (size_t)io * NC, b);
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    acc[0][j] = fma(d0, b[j], acc[0][j]);
                    acc[1][j] = fma(d1, b[j], acc[1][j]);
                }
            }
            const long long pt0 = (long long)((int)blockIdx.x + i * (int)gridDim.x) * kPtBM;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int ip = 4 * warp + q;
                if (ip >= np) break;
#pragma unroll
                for (int p = 0; p < 2; ++p) {
                    C v;
                    v.x = acc[p][2 * q];
                    v.y = acc[p][2 * q + 1];
                    planes[(size_t)ip * a.N + pt0 + lane + 32 * p] = v;
                }
            }
        }
        __syncthreads();  // the transposed tile is free for the next one
    }
    if (abort_flag && tid == 0) {
        atomicExch(err, 1);
        for (int i = 0; i < nmine; ++i)
            if (!mbar_try_wait(&full[i % kPtStages], (uint32_t)((i / kPtStages) & 1))) {
                (void)mbar_wait(&full[i % kPtStages], (uint32_t)((i / kPtStages) & 1));
                if (i + 1 < nmine) (void)mbar_wait(&full[(i + 1) % kPtStages], (uint32_t)(((i + 1) / kPtStages) & 1));
                break;
            }
    }
}

}  // namespace mdft
