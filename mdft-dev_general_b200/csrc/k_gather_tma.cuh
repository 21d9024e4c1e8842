// S7 gather fused with the ideal + external term (same arithmetic as k_gather), as a
// persistent pipeline: each resident CTA walks the tiles blockIdx.x, +gridDim.x, ...
// For each tile, warp 0 issues bulk copies of the tile's projection chunks (np runs of 32
// complex values), xi, vext and the search direction (three contiguous 32 x no runs of
// FP64) into one of two shared-memory stages; the copies of the next tile are in flight
// while the current one is computed.  The gamma -> orientation matrix B (2np x no) stays
// in shared memory for the whole launch.
//
// Tiles of BM points (32 for FP64, one CTA per SM; 16 for FP32, two CTAs per SM).  Warp w
// owns points PW w .. PW w + PW-1 (PW = BM/8) and lane l the orientations l, l+32, l+64
// (NCOL columns of 32), so the matrix products read the projections as broadcasts and B
// without bank conflicts, and each epilogue store of df is a coalesced 256-byte run.
// Partial sums (F_id, F_ext, F_exc sum, df.d, max|df|, sum w df) are kept per thread across tiles
// and reduced once per CTA in a fixed order.
//
// Used when N is a multiple of 32, no <= 96, the pointers are 16-byte aligned and the
// stages fit in shared memory (mmax <= 3); k_gather covers the rest.
#pragma once

#include "common.cuh"
#include "k_angular.cuh"
#include "k_fft.cuh"
#include "k_tma.cuh"

namespace mdft {

constexpr int kGtBM = 32;     // points per tile (FP64); FP32 uses kGtBM32 and two CTAs per SM
constexpr int kGtBM32 = 16;
constexpr int kGtStages = 2;  // pipeline depth
constexpr int kGtThreads = 256;

template <typename T> __host__ __device__ constexpr int gt_bm() { return sizeof(T) == 8 ? kGtBM : kGtBM32; }
template <typename T>
__host__ __device__ inline size_t gt_stage_bytes(int np, int no) {
    return (size_t)np * gt_bm<T>() * sizeof(typename Cplx<T>::t) + 3 * (size_t)gt_bm<T>() * no * sizeof(double);
}
template <typename T>
__host__ __device__ inline size_t gt_b_bytes(int np, int ncol) {
    return (size_t)2 * np * 32 * ncol * sizeof(T);
}
template <typename T>
inline size_t gather_tma_smem_bytes(int np, int no, int ncol) {
    return gt_b_bytes<T>(np, ncol) + kGtStages * gt_stage_bytes<T>(np, no);
}

// PW consecutive complex values from shared memory (PW*sizeof(C)-byte aligned)
template <int PW>
__device__ __forceinline__ void loadpw(const float2 *p, float2 (&v)[PW]) {
#pragma unroll
    for (int k = 0; k < PW; k += 2) {
        const float4 a = reinterpret_cast<const float4 *>(p)[k / 2];
        v[k] = make_float2(a.x, a.y);
        v[k + 1] = make_float2(a.z, a.w);
    }
}
template <int PW>
__device__ __forceinline__ void loadpw(const double2 *p, double2 (&v)[PW]) {
#pragma unroll
    for (int k = 0; k < PW; ++k) v[k] = p[k];
}

// TD: type of df and of the search direction (double, or float for the FP32 L-BFGS vectors);
// TX: type of xi and vext (double, or float in the FP32 phase of a mixed solve)
template <typename T, int NCOL, typename TD, typename TX = double>
__global__ void __launch_bounds__(kGtThreads, sizeof(T) == 8 ? 1 : 2) k_gather_tma(const typename Cplx<T>::t *__restrict__ planes,
                                                              const T *__restrict__ B, const TX *__restrict__ xi,
                                                              const TX *__restrict__ vext, const double *__restrict__ w,
                                                              TD *__restrict__ df, double *__restrict__ partial,
                                                              int *__restrict__ err, GatherArgs a, int ntiles) {
    using C = typename Cplx<T>::t;
    if (a.fail_wait) {  // the error path of a timed-out wait, with nothing issued yet
        if (threadIdx.x == 0) atomicExch(err, 1);
        return;
    }
    constexpr int NC = 32 * NCOL;
    constexpr int BM = gt_bm<T>();   // points per tile
    constexpr int PW = BM / 8;       // points per warp
    const int no = a.no, np = a.np, K = 2 * np;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    extern __shared__ __align__(128) unsigned char gt_smem[];
    T *Bs = reinterpret_cast<T *>(gt_smem);
    unsigned char *stage0 = gt_smem + gt_b_bytes<T>(np, NCOL);
    const size_t sbytes = gt_stage_bytes<T>(np, no);
    const size_t plbytes = (size_t)np * BM * sizeof(C);
    const size_t fbytes = (size_t)BM * no * sizeof(TX);
    __shared__ uint64_t full[kGtStages];
    __shared__ int abort_flag;
    __shared__ double red[kGatherSums][kGtThreads / 32];

    const bool want_v = a.do_ideal != 0, want_d = a.df_mode == 1 && a.dvec != nullptr;
    const size_t dbytes = (size_t)BM * no * sizeof(TD);
    const uint32_t tx = (uint32_t)(plbytes + fbytes * (1 + (want_v ? 1 : 0)) + (want_d ? dbytes : 0));
    const int nmine = (int)blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;

    auto issue = [&](int i) {  // warp 0: copies of this CTA's i-th tile into stage i % S
        const int s = i % kGtStages;
        const long long pt0 = (long long)((int)blockIdx.x + i * (int)gridDim.x) * BM;
        unsigned char *st = stage0 + s * sbytes;
        if (lane == 0) mbar_arrive_expect_tx(&full[s], tx);
        __syncwarp();
        const int ncopy = np + 3;
        for (int c = lane; c < ncopy; c += 32) {
            if (c < np) {
                bulk_load(st + (size_t)c * BM * sizeof(C), planes + (size_t)c * a.N + pt0, (uint32_t)(BM * sizeof(C)), &full[s]);
            } else if (c == np) {
                bulk_load(st + plbytes, xi + pt0 * no, (uint32_t)fbytes, &full[s]);
            } else if (c == np + 1) {
                if (want_v) bulk_load(st + plbytes + fbytes, vext + pt0 * no, (uint32_t)fbytes, &full[s]);
            } else {
                if (want_d)
                    bulk_load(st + plbytes + 2 * fbytes, static_cast<const TD *>(a.dvec) + pt0 * no, (uint32_t)dbytes, &full[s]);
            }
        }
    };

    if (tid == 0) {
        for (int s = 0; s < kGtStages; ++s) mbar_init(&full[s], 1);
        mbar_fence_init();
        abort_flag = 0;
    }
    __syncthreads();
    if (warp == 0)
        for (int i = 0; i < kGtStages && i < nmine; ++i) issue(i);
    // resident matrix, zero-padded to NC columns
    for (int f = tid; f < K * NC; f += kGtThreads) {
        const int k = f / NC, j = f % NC;
        Bs[f] = j < no ? B[(size_t)k * no + j] : (T)0;
    }
    double wv[NCOL];
#pragma unroll
    for (int c = 0; c < NCOL; ++c) wv[c] = (lane + 32 * c < no) ? w[lane + 32 * c] : 0.0;
    __syncthreads();

    const double pre = a.prefactor * a.cst;
    double fid = 0.0, fext = 0.0, fexc = 0.0, gdv = 0.0, gmx = 0.0, gun = 0.0;
    for (int i = 0; i < nmine; ++i) {
        const int s = i % kGtStages;
        const bool ok = mbar_wait(&full[s], (uint32_t)((i / kGtStages) & 1));
        if (!ok) abort_flag = 1;
        if (ok) {
            const unsigned char *st = stage0 + s * sbytes;
            const C *pl = reinterpret_cast<const C *>(st);
            const TX *xs = reinterpret_cast<const TX *>(st + plbytes);
            const TX *vs = xs + (size_t)BM * no;
            const TD *ds = reinterpret_cast<const TD *>(vs + (size_t)BM * no);
            T acc[PW][NCOL];
#pragma unroll
            for (int p = 0; p < PW; ++p)
#pragma unroll
                for (int c = 0; c < NCOL; ++c) acc[p][c] = (T)0;
#pragma unroll 4
            for (int ip = 0; ip < np; ++ip) {
                C av[PW];
                loadpw<PW>(pl + ip * BM + PW * warp, av);
                const T *br = Bs + (size_t)(2 * ip) * NC + lane;
#pragma unroll
                for (int c = 0; c < NCOL; ++c) {
                    const T bre = br[32 * c], bim = br[NC + 32 * c];
#pragma unroll
                    for (int p = 0; p < PW; ++p) {
                        acc[p][c] = fma(av[p].x, bre, acc[p][c]);
                        acc[p][c] = fma(av[p].y, bim, acc[p][c]);
                    }
                }
            }
            // Epilogue without branches on the data, so that the logs of a thread are
            // independent and interleave.  Columns past no have weight 0 and read a valid
            // element (e = 0); their results are not stored.  FP64 evaluations do the
            // per-element arithmetic in FP64; FP32 evaluations in FP32 (the pipeline's own
            // precision).  The sums are FP64 in both.
            const long long pt0 = (long long)((int)blockIdx.x + i * (int)gridDim.x) * BM;
#pragma unroll
            for (int p = 0; p < PW; ++p)
#pragma unroll
                for (int c = 0; c < NCOL; ++c) {
                    const int io = lane + 32 * c;
                    const bool valid = io < no;
                    const size_t e = valid ? (size_t)(PW * warp + p) * no + io : 0;
                    const T wio = (T)wv[c], r0 = (T)a.rho0;
                    const T vexc = (T)pre * wio * acc[p][c];
                    const T x = (T)xs[e];
                    const T x2 = x * x;
                    fexc += (double)((x2 * r0 - r0) * vexc);
                    const T dexc = (T)2 * r0 * x * vexc;
                    T did = (T)0;
                    if (want_v) {
                        const T v = (T)vs[e];
                        const T rho = x2 * r0;
                        const bool occ = (double)rho > kEpsDp;
                        const T lg = log(occ ? x2 : (T)1);  // log(rho / rho0)
                        const T kTdv = (T)(a.kT * a.dv), dv = (T)a.dv, kT = (T)a.kT;
                        fid += (double)(kTdv * wio * (occ ? rho * lg - rho + r0 : r0));
                        fext += occ ? (double)(dv * wio * rho * v) : 0.0;
                        did = occ ? wio * (T)2 * r0 * x * (kT * lg + v) : (T)0;
                    }
                    if (a.df_mode == 1) {
                        const double gv = (double)(did + dexc);
                        if (valid) df[pt0 * no + e] = (TD)gv;
                        if (want_d) gdv = fma(gv, (double)ds[e], gdv);
                        gmx = fmax(gmx, fabs(gv));
                        gun = fma(gv, wv[c], gun);
                    }
                }
        }
        __syncthreads();  // stage s fully consumed (and abort_flag visible)
        if (abort_flag) break;
        if (warp == 0 && i + kGtStages < nmine) issue(i + kGtStages);
    }
    if (abort_flag) {
        // A copy never completed: report it, then give the copies still in flight (the
        // failed tile's and, if issued, the next one's) a bounded wait before the CTA exits.
        if (tid == 0) {
            atomicExch(err, 1);
            for (int i = 0; i < nmine; ++i) {
                const bool done = mbar_try_wait(&full[i % kGtStages], (uint32_t)((i / kGtStages) & 1));
                if (!done) {
                    (void)mbar_wait(&full[i % kGtStages], (uint32_t)((i / kGtStages) & 1));
                    if (i + 1 < nmine) (void)mbar_wait(&full[(i + 1) % kGtStages], (uint32_t)(((i + 1) / kGtStages) & 1));
                    break;
                }
            }
        }
        return;
    }
    for (int off = 16; off > 0; off >>= 1) {
        fid += __shfl_down_sync(0xffffffffu, fid, off);
        fext += __shfl_down_sync(0xffffffffu, fext, off);
        fexc += __shfl_down_sync(0xffffffffu, fexc, off);
        gdv += __shfl_down_sync(0xffffffffu, gdv, off);
        gmx = fmax(gmx, __shfl_down_sync(0xffffffffu, gmx, off));
        gun += __shfl_down_sync(0xffffffffu, gun, off);
    }
    if (lane == 0) {
        red[0][warp] = fid;
        red[1][warp] = fext;
        red[2][warp] = fexc;
        red[3][warp] = gdv;
        red[4][warp] = gmx;
        red[5][warp] = gun;
    }
    __syncthreads();
    if (tid == 0) {
        double s0 = 0, s1 = 0, s2 = 0, s3 = 0, s4 = 0, s5 = 0;
        for (int k = 0; k < kGtThreads / 32; ++k) {
            s0 += red[0][k];
            s1 += red[1][k];
            s2 += red[2][k];
            s3 += red[3][k];
            s4 = fmax(s4, red[4][k]);
            s5 += red[5][k];
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

}  // namespace mdft
