// The angular contractions of the FP32 evaluations on the tcgen05 tensor cores, with
// split-BF16 operands: every FP32 operand v is carried as hi = bf16(v), lo = bf16(v - hi)
// and each product as hi*hi + hi*lo + lo*hi (three MMAs into one FP32 accumulator in tensor
// memory); the dropped lo*lo term and the two roundings leave a relative error near 2^-16
// per product.
//
//   S1, angl2proj (src/module_orientation_projection_transform.f90:159-199, restated as a
//   matrix product):  P[128 points x 2np] = drho[128 x no] . A[no x 2np],
//   drho = rho0 (xi^2 - 1)  ->  k_project_umma
//   S7, proj2angl + the ideal/external epilogue (src/module_energy_cproj_mrso.f90:728-762,
//   src/module_energy_ideal_and_external.f90:46-73):  V[128 x no] = P[128 x 2np] . B[2np x no]
//   ->  k_gather_umma
//
// One tile = 128 grid points (the MMA's M).  Each persistent CTA walks the tiles blockIdx.x,
// +gridDim.x, ...: all threads convert the tile's operand into the packed BF16 hi/lo layout
// of k_umma.cuh, thread 0 issues the MMAs and commits them to an mbarrier, every thread
// waits on it (bounded), and the epilogue reads the accumulator from tensor memory.  The
// angular matrix (hi and lo images, packed on the host) stays in shared memory for the
// launch.  Several CTAs per SM overlap one tile's loads with another's MMAs and stores.
// Used for mmax <= 3 (no <= 96, 2np <= 64) when N is a multiple of 128.
#pragma once

#include "common.cuh"
#include "k_angular.cuh"
#include "k_fft.cuh"
#include "k_umma.cuh"

namespace mdft {

constexpr int kUmBM = 128;       // points per tile (MMA M)
constexpr int kUmThreads = 256;  // 8 warps: two per tensor-memory lane quarter

struct UmmaShape {
    int Kp;     // reduction length padded to 16 (BF16 instruction K)
    int Np;     // output columns padded to 16
    int ncols;  // tensor-memory columns allocated (power of two >= Np, >= 32)
};

__host__ __device__ inline int round_up(int x, int m) { return (x + m - 1) / m * m; }
inline UmmaShape umma_shape(int K, int N) {
    UmmaShape s;
    s.Kp = round_up(K, 16);
    s.Np = round_up(N, 16);
    s.ncols = 32;
    while (s.ncols < s.Np) s.ncols *= 2;
    return s;
}
// shared memory: resident matrix (hi, lo) + the tile operand (hi, lo)
__host__ __device__ inline size_t umma_smem_bytes(const UmmaShape &s) {
    return 2 * umma::tile_bytes(s.Np, s.Kp, 2) + 2 * umma::tile_bytes(kUmBM, s.Kp, 2);
}
// extra shared memory of the gather: the accumulator tile as FP32 [128][no] and w(io)
inline size_t gather_umma_smem_bytes(const UmmaShape &s, int no) {
    return umma_smem_bytes(s) + (size_t)kUmBM * no * 4 + (size_t)round_up(no, 4) * 4;
}

// Shared set-up of both kernels: tensor memory, the mbarrier, the resident matrix.
struct UmmaCta {
    uint16_t *bhi, *blo, *ahi, *alo;
    uint32_t tmem;
};

__device__ __forceinline__ void umma_cta_setup(unsigned char *smem, const uint16_t *__restrict__ bimg, const UmmaShape &s,
                                               uint32_t *tmem_slot, uint64_t *bar, UmmaCta &c) {
    const int tid = threadIdx.x;
    const size_t bb = umma::tile_bytes(s.Np, s.Kp, 2), ab = umma::tile_bytes(kUmBM, s.Kp, 2);
    c.bhi = reinterpret_cast<uint16_t *>(smem);
    c.blo = reinterpret_cast<uint16_t *>(smem + bb);
    c.ahi = reinterpret_cast<uint16_t *>(smem + 2 * bb);
    c.alo = reinterpret_cast<uint16_t *>(smem + 2 * bb + ab);
    if ((tid >> 5) == 0) umma::tmem_alloc(tmem_slot, (uint32_t)s.ncols);
    if (tid == 0) {
        mbar_init(bar, 1);
        mbar_fence_init();
    }
    // the resident matrix: hi image then lo image, already in the packed layout
    const uint4 *src = reinterpret_cast<const uint4 *>(bimg);
    uint4 *dst = reinterpret_cast<uint4 *>(smem);
    for (size_t f = tid; f < 2 * bb / 16; f += blockDim.x) dst[f] = src[f];
    fence_proxy_async_smem();
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    c.tmem = *tmem_slot;
}

// Thread 0: the split-BF16 product of the tile (A hi/lo) with the resident matrix (B hi/lo)
// into tensor memory, then a commit to `bar`.
__device__ __forceinline__ void umma_issue(const UmmaCta &c, const UmmaShape &s, uint64_t *bar) {
    umma::fence_after_sync();
    const uint32_t sbo_a = (uint32_t)s.Kp * 16, sbo_b = sbo_a;  // (Kp / 8 chunks) x 128 bytes
    const uint32_t idesc = umma::instr_desc(1, s.Np);
    const uint32_t ah = smem_addr(c.ahi), al = smem_addr(c.alo), bh = smem_addr(c.bhi), bl = smem_addr(c.blo);
    for (int k = 0; k < s.Kp / 16; ++k) {
        const uint32_t off = (uint32_t)k * 256;  // 16 BF16 = two 128-byte core-matrix columns
        umma::mma<0>(c.tmem, umma::smem_desc(ah + off, sbo_a), umma::smem_desc(bh + off, sbo_b), idesc, k > 0);
        umma::mma<0>(c.tmem, umma::smem_desc(ah + off, sbo_a), umma::smem_desc(bl + off, sbo_b), idesc, true);
        umma::mma<0>(c.tmem, umma::smem_desc(al + off, sbo_a), umma::smem_desc(bh + off, sbo_b), idesc, true);
    }
    umma::commit(bar);
}

// Store 8 FP32 values as the hi and lo 16-byte chunks of row r, elements k0..k0+7.
__device__ __forceinline__ void store_split8(const UmmaCta &c, int Kp, int r, int k0, const float (&v)[8]) {
    uint32_t h[4], l[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) umma::split_bf16x2(v[2 * j], v[2 * j + 1], h[j], l[j]);
    const uint32_t off = umma::elem_offset(r, k0, Kp, 2);
    *reinterpret_cast<uint4 *>(reinterpret_cast<unsigned char *>(c.ahi) + off) = make_uint4(h[0], h[1], h[2], h[3]);
    *reinterpret_cast<uint4 *>(reinterpret_cast<unsigned char *>(c.alo) + off) = make_uint4(l[0], l[1], l[2], l[3]);
}

// ---------------------------------------------------------------------------------------
// S1: planes[ip][point] = sum_io drho(point, io) A(io, ip), drho = rho0 (xi^2 - 1).
// TX: type of xi (float in the FP32 phase of a mixed solve, double through the public API);
// VW: values per vector load of xi (4 when no % 4 == 0 and xi is 16-byte aligned, else 1).
// bimg: the packed hi and lo images of A^T ([Np][Kp]: row 2ip + {0: re, 1: im}, column io).
// The next tile's xi is loaded into registers while the current tile's MMAs and stores run.
constexpr int kPjThreads = 384;  // 12 warps, three per tensor-memory lane quarter; two CTAs per SM
constexpr int kPjTasks = (kUmBM * 12 + kPjThreads - 1) / kPjThreads;  // 128 points x (96 / 8) chunks

// v = x (FP32 xi) or x^2 - 1 formed in FP64 (FP64 xi) for the 8 orientations of each chunk
template <typename TX, int VW>
__device__ __forceinline__ void project_load(const TX *__restrict__ xi, long long pt0, int no, int KC, float (&v)[kPjTasks][8]) {
    const int tid = threadIdx.x;
#pragma unroll
    for (int q = 0; q < kPjTasks; ++q) {
        const int t = tid + q * kPjThreads;
        const int m = t % kUmBM, kc = t / kUmBM;
#pragma unroll
        for (int j = 0; j < 8; ++j) v[q][j] = 0.0f;
        if (kc >= KC) continue;
        const TX *row = xi + (pt0 + m) * no;
        const int k0 = 8 * kc;
        if (VW == 4 && k0 + 8 <= no) {
            if constexpr (sizeof(TX) == 4) {
                const float4 x0 = __ldg(reinterpret_cast<const float4 *>(row + k0));
                const float4 x1 = __ldg(reinterpret_cast<const float4 *>(row + k0) + 1);
                v[q][0] = x0.x; v[q][1] = x0.y; v[q][2] = x0.z; v[q][3] = x0.w;
                v[q][4] = x1.x; v[q][5] = x1.y; v[q][6] = x1.z; v[q][7] = x1.w;
            } else {
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const double2 x = __ldg(reinterpret_cast<const double2 *>(row + k0) + j);
                    v[q][2 * j] = (float)(x.x * x.x - 1.0);
                    v[q][2 * j + 1] = (float)(x.y * x.y - 1.0);
                }
            }
        } else {
#pragma unroll
            for (int j = 0; j < 8; ++j)
                if (k0 + j < no) {
                    const double x = (double)row[k0 + j];
                    v[q][j] = (sizeof(TX) == 4) ? (float)x : (float)(x * x - 1.0);
                }
        }
    }
}

template <typename TX>
__device__ __forceinline__ void project_store(const UmmaCta &c, int Kp, int no, int KC, float r0, const float (&v)[kPjTasks][8]) {
    const int tid = threadIdx.x;
#pragma unroll
    for (int q = 0; q < kPjTasks; ++q) {
        const int t = tid + q * kPjThreads;
        const int m = t % kUmBM, kc = t / kUmBM;
        if (kc >= KC) continue;
        float d[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            // FP32 xi: drho = rho0 (x^2 - 1) with one rounding of x^2 - 1 (fma)
            d[j] = (sizeof(TX) == 4) ? r0 * fmaf(v[q][j], v[q][j], -1.0f) : r0 * v[q][j];
            if (8 * kc + j >= no) d[j] = 0.0f;  // padding of the reduction
        }
        store_split8(c, Kp, m, 8 * kc, d);
    }
}

template <typename TX, int VW>
__global__ void __launch_bounds__(kPjThreads, 2) k_project_umma(const TX *__restrict__ xi, const uint16_t *__restrict__ bimg,
                                                                float2 *__restrict__ planes, int *__restrict__ err,
                                                                AngularArgs a, UmmaShape s, int ntiles) {
    extern __shared__ __align__(128) unsigned char um_smem[];
    __shared__ uint64_t bar;
    __shared__ uint32_t tmem_slot;
    __shared__ int abort_flag;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int no = a.no, np = a.np, KC = s.Kp / 8;
    if (tid == 0) abort_flag = 0;
    UmmaCta c;
    umma_cta_setup(um_smem, bimg, s, &tmem_slot, &bar, c);
    const float r0 = (float)a.rho0;
    const int nmine = (int)blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    auto tile0 = [&](int i) { return (long long)((int)blockIdx.x + i * (int)gridDim.x) * kUmBM; };
    float v[kPjTasks][8];
    if (nmine > 0) project_load<TX, VW>(xi, tile0(0), no, KC, v);
    int i = 0;  // after a failed wait: the tile whose MMA group may still run
    for (; i < nmine; ++i) {
        const long long pt0 = tile0(i);
        project_store<TX>(c, s.Kp, no, KC, r0, v);
        fence_proxy_async_smem();
        umma::fence_before_sync();
        __syncthreads();
        if (tid == 0) umma_issue(c, s, &bar);
        if (i + 1 < nmine) project_load<TX, VW>(xi, tile0(i + 1), no, KC, v);  // in flight during the MMAs
        if (!umma::wait_phase(&bar, (uint32_t)(i & 1))) abort_flag = 1;
        __syncthreads();  // every thread's wait result is in abort_flag: the branch below is uniform
        if (abort_flag) break;
        umma::fence_after_sync();
        // ---- epilogue: warp (quarter q4, third h) stores columns 16 cc .. 16 cc + 15, cc = h, h+3, ... ----
        const int q4 = warp & 3, h = warp >> 2;
        const long long pt = pt0 + 32 * q4 + lane;
        for (int cc = h; cc < s.Np / 16; cc += kPjThreads / 128) {
            float acc[16];
            umma::ld16(c.tmem + ((uint32_t)(32 * q4) << 16) + (uint32_t)(16 * cc), acc);
            umma::ld_wait();
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int ip = 8 * cc + j;
                if (ip < np) planes[(size_t)ip * a.N + pt] = make_float2(acc[2 * j], acc[2 * j + 1]);
            }
        }
        umma::fence_before_sync();  // tensor memory is rewritten by the next tile's MMAs after the next barrier
    }
    if (abort_flag && tid == 0) {
        atomicExch(err, 1);
        // the MMA group of the failed tile may still be running: give it a bounded wait
        (void)umma::wait_phase(&bar, (uint32_t)(i & 1));
    }
    __syncthreads();
    if (warp == 0) {
        umma::fence_after_sync();
        umma::tmem_free(c.tmem, (uint32_t)s.ncols);
    }
}

// ---------------------------------------------------------------------------------------
// S7 + ideal/external: V = P . B with P the tile's gamma projections (planes, FP32) and B
// the gamma -> orientation matrix; then per element, as k_gather_tma's FP32 epilogue:
// vexc = prefactor/N w V, F_exc += (x^2 rho0 - rho0) vexc, and with the ideal/external
// term F_id, F_ext, df = did + dexc, df.d, max|df|, sum w df (FP64 sums).
// TX: type of xi and vext; TD: type of df and of the search direction; NO: no when the
// element-wise epilogue runs on 4-element vectors (no % 4 == 0, compile-time modulo), else 0.
// bimg: the packed hi and lo images of B^T ([Np = no padded][Kp = 2np padded]).  The next
// tile's projections are loaded into registers while the current tile's MMAs and
// element-wise epilogue run.
constexpr int kGaTasks = 4;  // 128 points x (64 / 8) chunks over 256 threads

template <int NT = kUmThreads, int TASKS = kGaTasks>
__device__ __forceinline__ void gather_load(const float2 *__restrict__ planes, long long N, long long pt0, int np, int KC,
                                            float (&v)[TASKS][8]) {
    const int tid = threadIdx.x;
#pragma unroll
    for (int q = 0; q < TASKS; ++q) {
        const int t = tid + q * NT;
        const int m = t % kUmBM, kc = t / kUmBM;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int ip = 4 * kc + j;
            float2 p = make_float2(0.0f, 0.0f);
            if (kc < KC && ip < np) p = __ldg(planes + (size_t)ip * N + pt0 + m);
            v[q][2 * j] = p.x;
            v[q][2 * j + 1] = p.y;
        }
    }
}

template <typename T> __device__ __forceinline__ float4 ld4(const T *p);
template <> __device__ __forceinline__ float4 ld4<float>(const float *p) { return __ldg(reinterpret_cast<const float4 *>(p)); }
template <> __device__ __forceinline__ float4 ld4<double>(const double *p) {
    const double2 a = __ldg(reinterpret_cast<const double2 *>(p)), b = __ldg(reinterpret_cast<const double2 *>(p) + 1);
    return make_float4((float)a.x, (float)a.y, (float)b.x, (float)b.y);
}
// 4 elements of the direction in its own type (FP64 products with it in df.d)
template <typename T> struct Vec4T { T v[4]; };
template <typename T> __device__ __forceinline__ Vec4T<T> ld4t(const T *p);
template <> __device__ __forceinline__ Vec4T<float> ld4t<float>(const float *p) {
    const float4 a = __ldg(reinterpret_cast<const float4 *>(p));
    return Vec4T<float>{{a.x, a.y, a.z, a.w}};
}
template <> __device__ __forceinline__ Vec4T<double> ld4t<double>(const double *p) {
    const double2 a = __ldg(reinterpret_cast<const double2 *>(p)), b = __ldg(reinterpret_cast<const double2 *>(p) + 1);
    return Vec4T<double>{{a.x, a.y, b.x, b.y}};
}
template <typename T> __device__ __forceinline__ void st4(T *p, const double (&g)[4]);
template <> __device__ __forceinline__ void st4<float>(float *p, const double (&g)[4]) {
    *reinterpret_cast<float4 *>(p) = make_float4((float)g[0], (float)g[1], (float)g[2], (float)g[3]);
}
template <> __device__ __forceinline__ void st4<double>(double *p, const double (&g)[4]) {
    reinterpret_cast<double2 *>(p)[0] = make_double2(g[0], g[1]);
    reinterpret_cast<double2 *>(p)[1] = make_double2(g[2], g[3]);
}

// epsilon(1._dp) = 2^-52 as FP32 (exact): rho > kEpsDpF is the FP64 comparison of the reference
constexpr float kEpsDpF = 2.220446049250313080847263336181640625e-16f;

struct GatherConsts {
    float pre, r0, kT, dv, kTdv;
};

// One element of the FP32 epilogue (the arithmetic of k_gather_tma<float, ...>); returns df.
__device__ __forceinline__ float gather_elem(const GatherConsts &k, bool want_v, float acc, float wio, float x, float vv, double &fid,
                                             double &fext, double &fexc) {
    const float vexc = k.pre * wio * acc;
    const float x2 = x * x;
    fexc += (double)((x2 * k.r0 - k.r0) * vexc);
    const float dexc = 2.0f * k.r0 * x * vexc;
    float did = 0.0f;
    if (want_v) {
        const float rho = x2 * k.r0;
        const bool occ = rho > kEpsDpF;
        const float lg = logf(occ ? x2 : 1.0f);  // log(rho / rho0)
        fid += (double)(k.kTdv * wio * (occ ? rho * lg - rho + k.r0 : k.r0));
        fext += occ ? (double)(k.dv * wio * rho * vv) : 0.0;
        did = occ ? wio * 2.0f * k.r0 * x * (k.kT * lg + vv) : 0.0f;
    }
    return did + dexc;
}

// gather_elem with the element's terms added to FP32 accumulators (summed over a 4-element
// chunk before the FP64 accumulation)
__device__ __forceinline__ float gather_elem_f(const GatherConsts &k, bool want_v, float acc, float wio, float x, float vv, float &fid,
                                               float &fext, float &fexc) {
    const float vexc = k.pre * wio * acc;
    const float x2 = x * x;
    fexc += (x2 * k.r0 - k.r0) * vexc;
    const float dexc = 2.0f * k.r0 * x * vexc;
    float did = 0.0f;
    if (want_v) {
        const float rho = x2 * k.r0;
        const bool occ = rho > kEpsDpF;
        const float lg = logf(occ ? x2 : 1.0f);  // log(rho / rho0)
        fid += k.kTdv * wio * (occ ? rho * lg - rho + k.r0 : k.r0);
        fext += occ ? k.dv * wio * rho * vv : 0.0f;
        did = occ ? wio * 2.0f * k.r0 * x * (k.kT * lg + vv) : 0.0f;
    }
    return did + dexc;
}

template <typename TX, typename TD, int NO>
__global__ void __launch_bounds__(kUmThreads, 2) k_gather_umma(const float2 *__restrict__ planes, const uint16_t *__restrict__ bimg,
                                                               const TX *__restrict__ xi, const TX *__restrict__ vext,
                                                               const double *__restrict__ w, TD *__restrict__ df,
                                                               double *__restrict__ partial, int *__restrict__ err,
                                                               GatherArgs a, UmmaShape s, int ntiles) {
    if (a.fail_wait) {  // the error path of a timed-out wait, with nothing issued yet
        if (threadIdx.x == 0) atomicExch(err, 1);
        return;
    }
    extern __shared__ __align__(128) unsigned char um_smem[];
    __shared__ uint64_t bar;
    __shared__ uint32_t tmem_slot;
    __shared__ int abort_flag;
    __shared__ double red[kGatherSums][kUmThreads / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int no = NO > 0 ? NO : a.no, np = a.np, KC = s.Kp / 8;
    if (tid == 0) abort_flag = 0;
    UmmaCta c;
    umma_cta_setup(um_smem, bimg, s, &tmem_slot, &bar, c);
    float *vt = reinterpret_cast<float *>(um_smem + umma_smem_bytes(s));  // [128][no] accumulator tile
    float *ws = vt + (size_t)kUmBM * no;                                   // w(io), FP32
    for (int io = tid; io < no; io += kUmThreads) ws[io] = (float)w[io];
    __syncthreads();
    const bool want_v = a.do_ideal != 0, want_d = a.dvec != nullptr, store = a.df_mode == 1;
    const TD *dvec = static_cast<const TD *>(a.dvec);
    GatherConsts k;
    k.pre = (float)(a.prefactor * a.cst);
    k.r0 = (float)a.rho0;
    k.kT = (float)a.kT;
    k.dv = (float)a.dv;
    k.kTdv = (float)(a.kT * a.dv);
    const int nmine = (int)blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    auto tile0 = [&](int i) { return (long long)((int)blockIdx.x + i * (int)gridDim.x) * kUmBM; };
    double fid = 0.0, fext = 0.0, fexc = 0.0, gdv = 0.0, gmx = 0.0, gun = 0.0;
    float pv[kGaTasks][8];
    if (nmine > 0) gather_load(planes, a.N, tile0(0), np, KC, pv);
    int i = 0;  // after a failed wait: the tile whose MMA group may still run
    for (; i < nmine; ++i) {
        const long long pt0 = tile0(i);
#pragma unroll
        for (int q = 0; q < kGaTasks; ++q) {
            const int t = tid + q * kUmThreads;
            const int m = t % kUmBM, kc = t / kUmBM;
            if (kc < KC) store_split8(c, s.Kp, m, 8 * kc, pv[q]);
        }
        fence_proxy_async_smem();
        umma::fence_before_sync();
        __syncthreads();  // operand tile complete; the previous tile's epilogue is done with vt
        if (tid == 0) umma_issue(c, s, &bar);
        if (i + 1 < nmine) gather_load(planes, a.N, tile0(i + 1), np, KC, pv);  // in flight during the MMAs
        if (!umma::wait_phase(&bar, (uint32_t)(i & 1))) abort_flag = 1;
        __syncthreads();  // every thread's wait result is in abort_flag: the branch below is uniform
        if (abort_flag) break;
        umma::fence_after_sync();
        {
            // ---- accumulator -> shared [128][no] (row = point) ----
            const int q4 = warp & 3, h = warp >> 2;
            const int r = 32 * q4 + lane;
            for (int cc = h; cc < s.Np / 16; cc += 2) {
                float acc[16];
                umma::ld16(c.tmem + ((uint32_t)(32 * q4) << 16) + (uint32_t)(16 * cc), acc);
                umma::ld_wait();
                if (NO > 0) {
#pragma unroll
                    for (int j = 0; j < 16; j += 4) {
                        const int io = 16 * cc + j;
                        if (io < no)
                            *reinterpret_cast<float4 *>(vt + (size_t)r * no + io) = make_float4(acc[j], acc[j + 1], acc[j + 2], acc[j + 3]);
                    }
                } else {
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        const int io = 16 * cc + j;
                        if (io < no) vt[(size_t)r * no + io] = acc[j];
                    }
                }
            }
        }
        umma::fence_before_sync();
        __syncthreads();  // accumulator tile complete; tensor memory free for the next tile's MMAs
        // ---- element-wise epilogue over the tile's 128 x no values (coalesced) ----
        const long long e0 = pt0 * no;
        if constexpr (NO > 0) {
            static_assert(NO % 4 == 0, "vector epilogue needs no % 4 == 0");
            constexpr int NCH = kUmBM * NO / 4;  // 4-element chunks of the tile
            constexpr int U = 2;                 // chunks in flight per thread
            for (int cb = tid; cb < NCH; cb += U * kUmThreads) {
                float4 xv[U], vv[U];
                Vec4T<TD> dd[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int ch = cb + u * kUmThreads;
                    if (ch < NCH) {
                        xv[u] = ld4<TX>(xi + e0 + 4 * ch);
                        vv[u] = want_v ? ld4<TX>(vext + e0 + 4 * ch) : make_float4(0.f, 0.f, 0.f, 0.f);
                        if (want_d) dd[u] = ld4t<TD>(dvec + e0 + 4 * ch);
                    }
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int ch = cb + u * kUmThreads;
                    if (ch >= NCH) break;
                    const int io = (4 * ch) % NO;
                    const float4 av = *reinterpret_cast<const float4 *>(vt + 4 * ch);
                    const float4 wv = *reinterpret_cast<const float4 *>(ws + io);
                    double g[4];
                    g[0] = (double)gather_elem(k, want_v, av.x, wv.x, xv[u].x, vv[u].x, fid, fext, fexc);
                    g[1] = (double)gather_elem(k, want_v, av.y, wv.y, xv[u].y, vv[u].y, fid, fext, fexc);
                    g[2] = (double)gather_elem(k, want_v, av.z, wv.z, xv[u].z, vv[u].z, fid, fext, fexc);
                    g[3] = (double)gather_elem(k, want_v, av.w, wv.w, xv[u].w, vv[u].w, fid, fext, fexc);
                    if (store) {
                        st4<TD>(df + e0 + 4 * ch, g);
                        const float wj[4] = {wv.x, wv.y, wv.z, wv.w};
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            if (want_d) gdv = fma(g[j], (double)dd[u].v[j], gdv);
                            gmx = fmax(gmx, fabs(g[j]));
                            gun = fma(g[j], (double)wj[j], gun);
                        }
                    }
                }
            }
        } else {
            const int ne = kUmBM * no;
            for (int e = tid; e < ne; e += kUmThreads) {
                const int io = e % no;
                const float wio = ws[io];
                const float x = (float)xi[e0 + e];
                const float vv = want_v ? (float)vext[e0 + e] : 0.0f;
                const double gv = (double)gather_elem(k, want_v, vt[e], wio, x, vv, fid, fext, fexc);
                if (store) {
                    df[e0 + e] = (TD)gv;
                    if (want_d) gdv = fma(gv, (double)dvec[e0 + e], gdv);
                    gmx = fmax(gmx, fabs(gv));
                    gun = fma(gv, (double)wio, gun);
                }
            }
        }
    }
    if (abort_flag && tid == 0) {
        atomicExch(err, 1);
        (void)umma::wait_phase(&bar, (uint32_t)(i & 1));
    }
    __syncthreads();
    if (warp == 0) {
        umma::fence_after_sync();
        umma::tmem_free(c.tmem, (uint32_t)s.ncols);
    }
    if (abort_flag) return;
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
        for (int kk = 0; kk < kUmThreads / 32; ++kk) {
            s0 += red[0][kk];
            s1 += red[1][kk];
            s2 += red[2][kk];
            s3 += red[3][kk];
            s4 = fmax(s4, red[4][kk]);
            s5 += red[5][kk];
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

namespace mdft {

// ---------------------------------------------------------------------------------------
// Ring forms for the FP32 phase of mixed solves (FP32 point, vext, gradient and direction):
// one CTA per SM, with the tile data streamed by bulk copies (cp.async.bulk, no multicast)
// into a shared-memory ring ahead of use, so that HBM reads continue while the MMAs, the
// tensor-memory reads and the stores of a tile run.  Every mbarrier wait is bounded; after a
// failed wait thread 0 gives each copy and MMA group still outstanding a bounded wait, and
// the CTA frees its tensor memory and returns.

// Bounded waits on every phase still outstanding on a ring of barriers: issued[s] arrivals
// were asked of barrier s, done[s] of them have been waited for.
__device__ __forceinline__ void drain(uint64_t *bars, const int *issued, const int *done, int n) {
    for (int s = 0; s < n; ++s)
        for (int k = done[s]; k < issued[s]; ++k) (void)umma::wait_phase(&bars[s], (uint32_t)(k & 1));
}

// Shared-memory plan of k_project_ring: B hi/lo, two A hi/lo buffers, two x stages.
inline size_t project_ring_smem_bytes(const UmmaShape &s, int no) {
    return 2 * umma::tile_bytes(s.Np, s.Kp, 2) + 4 * umma::tile_bytes(kUmBM, s.Kp, 2) + 2 * (size_t)kUmBM * no * 4;
}

// S1 for an FP32 point: x tiles arrive by bulk copy two tiles ahead; the operand of tile i+1
// is converted (into the other A buffer) while the MMAs of tile i run, and the accumulators
// alternate between two tensor-memory column ranges.
constexpr int kRingThreads = 512;  // 16 warps: four per tensor-memory lane quarter

template <int VW>
__global__ void __launch_bounds__(kRingThreads, 1) k_project_ring(const float *__restrict__ xi, const uint16_t *__restrict__ bimg,
                                                                float2 *__restrict__ planes, int *__restrict__ err,
                                                                AngularArgs a, UmmaShape s, int ntiles) {
    extern __shared__ __align__(128) unsigned char um_smem[];
    __shared__ uint64_t xfull[2], mbar[2];
    __shared__ uint32_t tmem_slot;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int no = a.no, np = a.np, KC = s.Kp / 8;
    const size_t bb = umma::tile_bytes(s.Np, s.Kp, 2), ab = umma::tile_bytes(kUmBM, s.Kp, 2);
    const uint32_t xb = (uint32_t)(kUmBM * no * 4);
    uint16_t *bhi = reinterpret_cast<uint16_t *>(um_smem), *blo = reinterpret_cast<uint16_t *>(um_smem + bb);
    unsigned char *abuf = um_smem + 2 * bb;                         // A[k] hi at abuf + 2k ab, lo at + ab
    float *xs = reinterpret_cast<float *>(um_smem + 2 * bb + 4 * ab);  // x stage k at xs + k kUmBM no
    const uint32_t ncols = (uint32_t)s.ncols * 2;                     // two accumulator column ranges
    if (warp == 0) umma::tmem_alloc(&tmem_slot, ncols);
    if (tid == 0) {
        for (int k = 0; k < 2; ++k) {
            mbar_init(&xfull[k], 1);
            mbar_init(&mbar[k], 1);
        }
        mbar_fence_init();
    }
    {
        const uint4 *src = reinterpret_cast<const uint4 *>(bimg);
        uint4 *dst = reinterpret_cast<uint4 *>(um_smem);
        for (size_t f = tid; f < 2 * bb / 16; f += blockDim.x) dst[f] = src[f];
    }
    fence_proxy_async_smem();
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = tmem_slot;
    const int nmine = (int)blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    auto tile0 = [&](int i) { return (long long)((int)blockIdx.x + i * (int)gridDim.x) * kUmBM; };
    // thread 0's bookkeeping of the barriers, for the bounded drain after a failed wait
    int xiss[2] = {0, 0}, xdone[2] = {0, 0}, miss[2] = {0, 0}, mdone[2] = {0, 0};
    auto copy_x = [&](int i) {  // thread 0
        const int k = i & 1;
        mbar_arrive_expect_tx(&xfull[k], xb);
        bulk_load(xs + (size_t)k * kUmBM * no, xi + tile0(i) * no, xb, &xfull[k]);
        ++xiss[k];
    };
    // x stage (i & 1) -> A buffer (i & 1), split BF16; false when the copy's wait ran out
    auto convert = [&](int i) -> bool {
        const int k = i & 1;
        const bool ok = umma::wait_phase(&xfull[k], (uint32_t)((i >> 1) & 1));
        if (!ok) return false;
        if (tid == 0) ++xdone[k];
        const float *x = xs + (size_t)k * kUmBM * no;
        UmmaCta c;
        c.ahi = reinterpret_cast<uint16_t *>(abuf + 2 * k * ab);
        c.alo = reinterpret_cast<uint16_t *>(abuf + (2 * k + 1) * ab);
        const float r0 = (float)a.rho0;
        for (int t = tid; t < kUmBM * KC; t += kRingThreads) {
            const int m = t % kUmBM, kc = t / kUmBM, k0 = 8 * kc;
            const float *row = x + m * no;
            float v[8];
            if (VW == 4 && k0 + 8 <= no) {
                const float4 x0 = reinterpret_cast<const float4 *>(row + k0)[0], x1 = reinterpret_cast<const float4 *>(row + k0)[1];
                v[0] = x0.x; v[1] = x0.y; v[2] = x0.z; v[3] = x0.w; v[4] = x1.x; v[5] = x1.y; v[6] = x1.z; v[7] = x1.w;
            } else {
#pragma unroll
                for (int j = 0; j < 8; ++j) v[j] = (k0 + j < no) ? row[k0 + j] : 1.0f;
            }
#pragma unroll
            for (int j = 0; j < 8; ++j) v[j] = (k0 + j < no) ? r0 * fmaf(v[j], v[j], -1.0f) : 0.0f;
            store_split8(c, s.Kp, m, k0, v);
        }
        return true;
    };
    auto issue = [&](int i) {  // thread 0: MMAs of tile i into column range (i & 1)
        const int k = i & 1;
        UmmaCta c;
        c.bhi = bhi;
        c.blo = blo;
        c.ahi = reinterpret_cast<uint16_t *>(abuf + 2 * k * ab);
        c.alo = reinterpret_cast<uint16_t *>(abuf + (2 * k + 1) * ab);
        c.tmem = tmem + (uint32_t)(k * s.ncols);
        umma_issue(c, s, &mbar[k]);
        ++miss[k];
    };
    if (tid == 0)
        for (int i = 0; i < 2 && i < nmine; ++i) copy_x(i);
    // prologue: tile 0's operand and MMAs.  A failed wait anywhere in the block is seen by
    // every thread through the barrier's OR (aborted stays uniform).
    bool aborted = false;
    if (nmine > 0) {
        const bool ok = convert(0);
        fence_proxy_async_smem();
        umma::fence_before_sync();
        aborted = __syncthreads_or(!ok) != 0;
        if (!aborted && tid == 0) {
            if (2 < nmine) copy_x(2);
            issue(0);
        }
    }
    for (int i = 0; i < nmine && !aborted; ++i) {
        // the next tile's operand while this tile's MMAs run
        if (i + 1 < nmine) {
            const bool ok = convert(i + 1);
            fence_proxy_async_smem();
            umma::fence_before_sync();
            if (__syncthreads_or(!ok)) { aborted = true; break; }
            if (tid == 0) {
                if (i + 3 < nmine) copy_x(i + 3);
                issue(i + 1);
            }
        }
        const bool ok = umma::wait_phase(&mbar[i & 1], (uint32_t)((i >> 1) & 1));
        if (tid == 0 && ok) ++mdone[i & 1];
        if (__syncthreads_or(!ok)) { aborted = true; break; }
        umma::fence_after_sync();
        const int q4 = warp & 3, h = warp >> 2;
        const long long pt = tile0(i) + 32 * q4 + lane;
        const uint32_t cbase = tmem + ((uint32_t)(32 * q4) << 16) + (uint32_t)((i & 1) * s.ncols);
        for (int cc = h; cc < s.Np / 16; cc += kRingThreads / 128) {
            float acc[16];
            umma::ld16(cbase + (uint32_t)(16 * cc), acc);
            umma::ld_wait();
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int ip = 8 * cc + j;
                if (ip < np) planes[(size_t)ip * a.N + pt] = make_float2(acc[2 * j], acc[2 * j + 1]);
            }
        }
        umma::fence_before_sync();
    }
    __syncthreads();
    if (aborted && tid == 0) {
        atomicExch(err, 1);
        drain(xfull, xiss, xdone, 2);
        drain(mbar, miss, mdone, 2);
    }
    __syncthreads();
    if (warp == 0) {
        umma::fence_after_sync();
        umma::tmem_free(tmem, ncols);
    }
}

// Shared-memory plan of k_gather_ring: B hi/lo, A hi/lo, the accumulator tile [128][NO],
// and kGrStages stages of one 32-point sub-tile of x, vext and the direction.
constexpr int kGrStages = 3;
constexpr int kGrSub = 32;                 // points per streamed sub-tile
constexpr int kGrPer = kUmBM / kGrSub;     // sub-tiles per tile
// one thread per 4-orientation chunk of a sub-tile: every thread has the same work per stage
template <int NO> __host__ __device__ constexpr int gather_ring_threads() { return kGrSub * NO / 4; }
// the block: those threads plus one copy warp
template <int NO> __host__ __device__ constexpr int gather_ring_block() { return gather_ring_threads<NO>() + 32; }
inline size_t gather_ring_smem_bytes(const UmmaShape &s, int no) {
    // + the projections of one tile, [Kp / 2 complex][128 points]
    return umma_smem_bytes(s) + (size_t)kUmBM * no * 4 + (size_t)kGrStages * 3 * kGrSub * no * 4 + (size_t)(s.Kp / 2) * kUmBM * 8;
}

// log(v) for the ring epilogue: the hardware base-2 logarithm (lg2.approx; absolute error
// about 2^-22 in log2, below the FP32 rounding of the other terms of df) times ln 2.  v is
// x^2 > eps / rho0 or 1, never subnormal.
__device__ __forceinline__ float ring_log(float v) {
    float r;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(v));
    return r * 0.693147180559945309417232121458176568f;
}

// S7 + ideal/external for the FP32 phase (x, vext, df, direction all FP32; NO % 4 == 0).
// Warp specialised: a copy warp streams x, vext and the direction of each 32-point sub-tile
// by bulk copy into a kGrStages ring, refilling a stage as soon as every epilogue warp has
// arrived on its "empty" barrier; the epilogue warps (one thread per 4-orientation chunk of a
// sub-tile: point 4t / NO, orientations 4t % NO .., w(io) in registers) load the projections
// of the next tile into registers while the current tile's MMAs run, and synchronise among
// themselves only three times per 128-point tile (named barrier 1), not per sub-tile.
//
// Per element (x, vext v, accumulator a = sum_ip conj-product, weight w):
//   occ = rho0 x^2 > eps;  lg = log x^2 (occ)
//   df  = 2 rho0 w x (pre a + [occ] (kT lg + v))
//   F_exc term = pre rho0 w a (x^2 - 1);  F_id term = kT dv rho0 w ([occ] x^2 (lg - 1) + 1);
//   F_ext term = dv rho0 [occ] w x^2 v
// (the arithmetic of gather_elem with the constant factors taken out of the sums; the
// constant part of F_id, kT dv rho0 sum w, is added per tile in FP64).
template <int NO>
__global__ void __launch_bounds__(gather_ring_block<NO>(), 1) k_gather_ring(const float2 *__restrict__ planes, const uint16_t *__restrict__ bimg,
                                                               const float *__restrict__ xi, const float *__restrict__ vext,
                                                               const double *__restrict__ w, float *__restrict__ df,
                                                               double *__restrict__ partial, int *__restrict__ err,
                                                               GatherArgs a, UmmaShape s, int ntiles) {
    static_assert(NO % 4 == 0, "vector epilogue needs no % 4 == 0");
    if (a.fail_wait) {  // the error path of a timed-out wait, with nothing issued yet
        if (threadIdx.x == 0) atomicExch(err, 1);
        return;
    }
    constexpr int NT = gather_ring_threads<NO>();  // epilogue threads
    static_assert(NT % 32 == 0, "whole warps");
    static_assert(NT + 32 <= 1024, "one CTA of at most 1024 threads");
    constexpr int kWarps = NT / 32 + 1, kGroupWarps = (NT / 32) / 4;  // epilogue warps per tensor-memory lane quarter
    constexpr uint32_t kEpiBar = 1;                                   // named barrier of the epilogue threads
    extern __shared__ __align__(128) unsigned char um_smem[];
    __shared__ uint64_t bar, sfull[kGrStages], sempty[kGrStages], pfull, pempty;
    __shared__ uint32_t tmem_slot;
    __shared__ double red[kGatherSums][kWarps];
    __shared__ double wsum_s;
    __shared__ int abort_s;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const bool copier = tid >= NT;
    const int np = a.np, KC = s.Kp / 8;
    constexpr int kTasks = (kUmBM * 8 + NT - 1) / NT;  // 8-element chunks of the P tile per thread (Kp <= 64)
    if (tid == 0) {
        for (int k = 0; k < kGrStages; ++k) {
            mbar_init(&sfull[k], 1);
            mbar_init(&sempty[k], NT / 32);
        }
        mbar_init(&pfull, 1);
        mbar_init(&pempty, NT / 32);
        double ws = 0.0;
        for (int io = 0; io < NO; ++io) ws += w[io];
        wsum_s = ws;
        abort_s = 0;
    }
    UmmaCta c;
    umma_cta_setup(um_smem, bimg, s, &tmem_slot, &bar, c);  // also fences the barrier inits (block barrier)
    float *vt = reinterpret_cast<float *>(um_smem + umma_smem_bytes(s));  // [128][NO]
    float *ring = vt + (size_t)kUmBM * NO;  // stage k: x, vext, d of kGrSub points each
    constexpr int SUB = kGrSub * NO;        // floats per array per sub-tile
    float2 *pst = reinterpret_cast<float2 *>(ring + (size_t)kGrStages * 3 * SUB);  // [np][128] of the next tile
    const bool want_v = a.do_ideal != 0, want_d = a.dvec != nullptr, store = a.df_mode == 1;
    const float *dvec = static_cast<const float *>(a.dvec);
    const int nmine = (int)blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    const int nsub = kGrPer * nmine;
    auto tile0 = [&](int i) { return (long long)((int)blockIdx.x + i * (int)gridDim.x) * kUmBM; };
    double fid = 0.0, fext = 0.0, fexc = 0.0, gdv = 0.0, gmx = 0.0, gun = 0.0;
    bool aborted = false;
    if (copier) {
        // ---- the copy warp: sub-tile G into stage G % kGrStages once the stage is empty ----
        const uint32_t sb = (uint32_t)(SUB * 4);
        const uint32_t tx = sb * (1u + (want_v ? 1u : 0u) + (want_d ? 1u : 0u));
        const uint32_t pb = (uint32_t)(kUmBM * sizeof(float2));  // one projection of a tile
        int issued[kGrStages] = {}, pissued = 0;
        for (int G = 0; G < nsub; ++G) {
            const int st = G % kGrStages;
            if (G % kGrPer == 0) {
                // tile G / kGrPer's projections, once the previous tile's are in the A tile
                const int i = G / kGrPer;
                if (i > 0 && !mbar_wait(&pempty, (uint32_t)((i - 1) & 1))) {
                    aborted = true;
                    break;
                }
                if (lane == 0) {
                    mbar_arrive_expect_tx(&pfull, pb * (uint32_t)np);
                    for (int ip = 0; ip < np; ++ip) bulk_load(pst + (size_t)ip * kUmBM, planes + (size_t)ip * a.N + tile0(i), pb, &pfull);
                }
                ++pissued;
            }
            if (G >= kGrStages && !mbar_wait(&sempty[st], (uint32_t)((G / kGrStages - 1) & 1))) {
                aborted = true;  // the epilogue warps stopped (or stalled): copy nothing more
                break;
            }
            if (lane == 0) {
                const long long e = (tile0(G / kGrPer) + (long long)kGrSub * (G % kGrPer)) * NO;
                float *dst = ring + (size_t)st * 3 * SUB;
                mbar_arrive_expect_tx(&sfull[st], tx);
                bulk_load(dst, xi + e, sb, &sfull[st]);
                if (want_v) bulk_load(dst + SUB, vext + e, sb, &sfull[st]);
                if (want_d) bulk_load(dst + 2 * SUB, dvec + e, sb, &sfull[st]);
            }
            ++issued[st];
        }
        // every copy issued has landed (or had its bounded wait) before the block ends
        if (lane == 0) {
            for (int st = 0; st < kGrStages; ++st)
                if (issued[st] > 0) (void)mbar_wait(&sfull[st], (uint32_t)((issued[st] - 1) & 1));
            if (pissued > 0) (void)mbar_wait(&pfull, (uint32_t)((pissued - 1) & 1));
        }
        if (aborted && lane == 0) atomicExch(err, 1);
    } else {
        // ---- the epilogue warps ----
        const float pre = (float)(a.prefactor * a.cst), kT = (float)a.kT;
        const float er0 = (float)(2.220446049250313080847263336181640625e-16 / a.rho0);  // rho0 x^2 > eps
        const int io0 = (4 * tid) % NO;
        float wv[4], w2v[4];  // w(io) and 2 rho0 w(io) of this thread's orientations
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            wv[u] = (float)w[io0 + u];
            w2v[u] = (float)(2.0 * a.rho0 * w[io0 + u]);
        }
        const double cid = a.kT * a.dv * a.rho0, cext = a.dv * a.rho0, cexc = (double)pre * a.rho0;
        const double tile_id = want_v ? cid * (double)kUmBM * wsum_s : 0.0;  // constant part of F_id per tile
        int miss = 0, mdone = 0;  // thread 0's MMA bookkeeping
        bool lost = false;  // this thread saw a copy that did not land in time
        for (int i = 0; i < nmine; ++i) {
            // the tile's projections (staged by the copy warp) split into the A tile
            const bool okp = !lost && umma::wait_phase(&pfull, (uint32_t)(i & 1));
            if (!okp) lost = true;
#pragma unroll
            for (int q = 0; q < kTasks; ++q) {
                const int t = tid + q * NT;
                const int m = t % kUmBM, kc = t / kUmBM;
                if (kc < KC) {
                    float v[8];
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const int ip = 4 * kc + j;
                        const float2 p = (okp && ip < np) ? pst[(size_t)ip * kUmBM + m] : make_float2(0.f, 0.f);
                        v[2 * j] = p.x;
                        v[2 * j + 1] = p.y;
                    }
                    store_split8(c, s.Kp, m, 8 * kc, v);
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&pempty);  // this warp is done with the staged projections
            fence_proxy_async_smem();
            umma::fence_before_sync();
            named_sync(kEpiBar, NT);
            if (tid == 0) {
                umma_issue(c, s, &bar);
                ++miss;
            }
            const bool ok = umma::wait_phase(&bar, (uint32_t)(i & 1));
            if (tid == 0 && ok) ++mdone;
            // one agreement per tile: an MMA or a copy that did not complete stops every epilogue warp
            if (named_sync_or(kEpiBar, NT, !ok || lost)) {
                aborted = true;
                break;
            }
            umma::fence_after_sync();
            if (warp < 4 * kGroupWarps) {
                const int q4 = warp & 3, h = warp >> 2;
                const int r = 32 * q4 + lane;
                for (int cc = h; cc < s.Np / 16; cc += kGroupWarps) {
                    float acc[16];
                    umma::ld16(c.tmem + ((uint32_t)(32 * q4) << 16) + (uint32_t)(16 * cc), acc);
                    umma::ld_wait();
#pragma unroll
                    for (int j = 0; j < 16; j += 4) {
                        const int io = 16 * cc + j;
                        if (io < NO) *reinterpret_cast<float4 *>(vt + (size_t)r * NO + io) = make_float4(acc[j], acc[j + 1], acc[j + 2], acc[j + 3]);
                    }
                }
            }
            umma::fence_before_sync();
            named_sync(kEpiBar, NT);  // accumulator tile complete; tensor memory free for the next tile's MMAs
            // the tile's terms of each sum in FP32 (kGrPer * 4 per thread), then one FP64 addition
            // per sum: the FP32 -> FP64 conversions stay off the per-element path
            float tid_ = 0.f, text = 0.f, texc = 0.f, tgd = 0.f, tgm = 0.f, tgu = 0.f;
            for (int j = 0; j < kGrPer; ++j) {
                const int G = kGrPer * i + j, st = G % kGrStages;
                const bool okc = !lost && umma::wait_phase(&sfull[st], (uint32_t)((G / kGrStages) & 1));
                if (okc) {
                    const float *xsv = ring + (size_t)st * 3 * SUB, *vsv = xsv + SUB, *dsv = xsv + 2 * SUB;
                    const float *acc = vt + (size_t)kGrSub * j * NO;
                    const float4 x4 = reinterpret_cast<const float4 *>(xsv)[tid];
                    const float4 v4 = want_v ? reinterpret_cast<const float4 *>(vsv)[tid] : make_float4(0.f, 0.f, 0.f, 0.f);
                    const float4 a4 = reinterpret_cast<const float4 *>(acc)[tid];
                    const float xs[4] = {x4.x, x4.y, x4.z, x4.w}, vs[4] = {v4.x, v4.y, v4.z, v4.w}, as[4] = {a4.x, a4.y, a4.z, a4.w};
                    float g[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const float x = xs[u], x2 = x * x;
                        const bool occ = want_v && x2 > er0;
                        const float lg = ring_log(occ ? x2 : 1.0f);
                        const float wx2 = occ ? wv[u] * x2 : 0.0f;
                        tid_ = fmaf(wx2, lg - 1.0f, tid_);
                        text = fmaf(wx2, vs[u], text);
                        const float inner = occ ? fmaf(kT, lg, vs[u]) : 0.0f;
                        g[u] = (w2v[u] * x) * fmaf(pre, as[u], inner);
                        texc = fmaf(wv[u] * as[u], fmaf(x, x, -1.0f), texc);
                    }
                    if (store) {
                        const long long e0 = (tile0(i) + (long long)kGrSub * j) * NO;
                        *reinterpret_cast<float4 *>(df + e0 + 4 * tid) = make_float4(g[0], g[1], g[2], g[3]);
                        if (want_d) {
                            const float4 dd = reinterpret_cast<const float4 *>(dsv)[tid];
                            tgd = fmaf(g[0], dd.x, fmaf(g[1], dd.y, fmaf(g[2], dd.z, fmaf(g[3], dd.w, tgd))));
                        }
                        tgm = fmaxf(tgm, fmaxf(fmaxf(fabsf(g[0]), fabsf(g[1])), fmaxf(fabsf(g[2]), fabsf(g[3]))));
                        tgu = fmaf(g[0], wv[0], fmaf(g[1], wv[1], fmaf(g[2], wv[2], fmaf(g[3], wv[3], tgu))));
                    }
                } else {
                    lost = true;
                }
                // this warp is done with stage st (its reads are complete before the arrival)
                __syncwarp();
                if (lane == 0) mbar_arrive(&sempty[st]);
            }
            if (tid == 0) fid += tile_id;
            fid += cid * (double)tid_;
            fext += cext * (double)text;
            fexc += cexc * (double)texc;
            gdv += (double)tgd;
            gmx = fmax(gmx, (double)tgm);
            gun += (double)tgu;
        }
        if (!aborted && named_sync_or(kEpiBar, NT, lost)) aborted = true;  // a copy lost in the last tile
        if (aborted && tid == 0) {
            atomicExch(err, 1);
            drain(&bar, &miss, &mdone, 1);
        }
    }
    if (aborted) abort_s = 1;  // benign race: every writer stores 1
    __syncthreads();
    if (warp == 0) {
        umma::fence_after_sync();
        umma::tmem_free(c.tmem, (uint32_t)s.ncols);
    }
    if (abort_s) return;
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
        for (int kk = 0; kk < kWarps; ++kk) {
            s0 += red[0][kk];
            s1 += red[1][kk];
            s2 += red[2][kk];
            s3 += red[3][kk];
            s4 = fmax(s4, red[4][kk]);
            s5 += red[5][kk];
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
