// Batched 3-D FFTs over the projection planes, templated on precision and length.
//
//  k_fft_xy<T, N>  : one CTA per (projection, z) plane of N x N points: the plane is
//                    staged in shared memory, transformed along x then y, written back.
//  k_fft_z<T, N>   : one CTA per (projection, y) and TL consecutive x: columns along z.
//
// Every radix pass is in place: each thread loads the inputs of its butterflies into
// registers (twiddled), a barrier, then writes the outputs at their Stockham positions.
// The radix sequence (4s, then 2, then 3s) is fixed at compile time, so butterflies are
// fully unrolled.  sign=+1: X[k] = sum_j x[j] e^{+2 pi i jk/N} (plan3dp of
// src/module_energy_cproj_mrso.f90:260); sign=-1: plan3dm; no scaling.
#pragma once

#include "common.cuh"
#include "k_fft.cuh"
#include "k_tma.cuh"

namespace mdft {

__host__ __device__ constexpr int count_factor(int n, int f) { return (n % f == 0 && n > 1) ? 1 + count_factor(n / f, f) : 0; }
__host__ __device__ constexpr int ipow(int b, int e) { return e == 0 ? 1 : b * ipow(b, e - 1); }
// passes of length n: all radix-8 passes, then 4s, 2s and 3s on what is left
__host__ __device__ constexpr int n8_of(int n) { return count_factor(n, 8); }
__host__ __device__ constexpr int r8_of(int n) { return n / ipow(8, n8_of(n)); }  // the part after the 8s
__host__ __device__ constexpr int n4_of(int n) { return count_factor(r8_of(n), 4); }
__host__ __device__ constexpr int n2_of(int n) { return count_factor(r8_of(n) / ipow(4, n4_of(n)), 2); }
__host__ __device__ constexpr int n3_of(int n) { return count_factor(r8_of(n) / ipow(4, n4_of(n)) / ipow(2, n2_of(n)), 3); }
__host__ __device__ constexpr int npass_of(int n) { return n8_of(n) + n4_of(n) + n2_of(n) + n3_of(n); }
// radix of pass p for length n: all 8s, then 4s, 2s, 3s
__host__ __device__ constexpr int radix_of(int n, int p) {
    return p < n8_of(n) ? 8 : p < n8_of(n) + n4_of(n) ? 4 : p < n8_of(n) + n4_of(n) + n2_of(n) ? 2 : 3;
}
// product of the radices before pass p (the Stockham span Ns)
__host__ __device__ constexpr int span_of(int n, int p) { return p == 0 ? 1 : span_of(n, p - 1) * radix_of(n, p - 1); }

template <typename T, int R>
__device__ __forceinline__ void dft_small(typename Cplx<T>::t (&v)[R], int sign) {
    using C = typename Cplx<T>::t;
    if constexpr (R == 2) {
        C a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    } else if constexpr (R == 4) {
        C s02 = cadd(v[0], v[2]), d02 = csub(v[0], v[2]);
        C s13 = cadd(v[1], v[3]), d13 = csub(v[1], v[3]);
        C wd;
        wd.x = -(T)sign * d13.y;
        wd.y = (T)sign * d13.x;
        v[0] = cadd(s02, s13);
        v[1] = cadd(d02, wd);
        v[2] = csub(s02, s13);
        v[3] = csub(d02, wd);
    } else if constexpr (R == 8) {
        // radix 2 between j and j + 4, twiddles w^j (w = e^{sign 2 pi i / 8}), then two radix-4
        // DFTs: the even outputs from the sums, the odd outputs from the twiddled differences
        const T h = (T)0.70710678118654752440084436210484903928;
        C a[4], b[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            a[j] = cadd(v[j], v[j + 4]);
            b[j] = csub(v[j], v[j + 4]);
        }
        const T sg = (T)sign;
        // b1 *= (1 + i sg)/sqrt2, b2 *= i sg, b3 *= (-1 + i sg)/sqrt2
        C t;
        t.x = h * (b[1].x - sg * b[1].y);
        t.y = h * (b[1].y + sg * b[1].x);
        b[1] = t;
        t.x = -sg * b[2].y;
        t.y = sg * b[2].x;
        b[2] = t;
        t.x = h * (-b[3].x - sg * b[3].y);
        t.y = h * (-b[3].y + sg * b[3].x);
        b[3] = t;
        dft_small<T, 4>(a, sign);
        dft_small<T, 4>(b, sign);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            v[2 * k] = a[k];
            v[2 * k + 1] = b[k];
        }
    } else {  // R == 3
        const T c3 = (T)-0.5;
        const T s3 = (T)sign * (T)0.86602540378443864676372317075294;
        C s12 = cadd(v[1], v[2]), d12 = csub(v[1], v[2]);
        C m;
        m.x = v[0].x + c3 * s12.x;
        m.y = v[0].y + c3 * s12.y;
        C rot;
        rot.x = -s3 * d12.y;
        rot.y = s3 * d12.x;
        v[0] = cadd(v[0], s12);
        v[1] = cadd(m, rot);
        v[2] = csub(m, rot);
    }
}

// One in-place Stockham pass of radix R over `lines` transforms of length N stored at
// buf[line * lstride + i * istride]; tw[t] = e^{+2 pi i t/N}.  LF: consecutive threads take
// consecutive lines (for strided lines, so that shared-memory accesses stay contiguous).
template <typename T, int N, int R, int NS, int LINES, int THREADS, bool LF>
__device__ __forceinline__ void stockham_pass(typename Cplx<T>::t *buf, int istride, int lstride,
                                              const typename Cplx<T>::t *tw, int sign) {
    using C = typename Cplx<T>::t;
    constexpr int NB = N / R;
    constexpr int ITEMS = NB * LINES;
    constexpr int PER = (ITEMS + THREADS - 1) / THREADS;
    constexpr int TSTEP = N / (NS * R);
    C v[PER][R];
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        const int it = threadIdx.x + k * THREADS;
        if (ITEMS % THREADS == 0 || it < ITEMS) {
            const int line = LF ? it % LINES : it / NB, j = LF ? it / LINES : it % NB, jm = j % NS;
            C *b = buf + line * lstride;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                C x = b[(j + r * NB) * istride];
                if (r > 0 && NS > 1) {
                    C w = tw[(jm * TSTEP * r) % N];
                    if (sign < 0) w.y = -w.y;
                    x = cmul(x, w);
                }
                v[k][r] = x;
            }
            dft_small<T, R>(v[k], sign);
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        const int it = threadIdx.x + k * THREADS;
        if (ITEMS % THREADS == 0 || it < ITEMS) {
            const int line = LF ? it % LINES : it / NB, j = LF ? it / LINES : it % NB, jm = j % NS;
            C *b = buf + line * lstride;
            const int idxD = (j / NS) * NS * R + jm;
#pragma unroll
            for (int r = 0; r < R; ++r) b[(idxD + r * NS) * istride] = v[k][r];
        }
    }
    __syncthreads();
}

template <typename T, int N, int P, int LINES, int THREADS, bool LF>
__device__ __forceinline__ void fft_lines(typename Cplx<T>::t *buf, int istride, int lstride,
                                          const typename Cplx<T>::t *tw, int sign) {
    if constexpr (P < npass_of(N)) {
        stockham_pass<T, N, radix_of(N, P), span_of(N, P), LINES, THREADS, LF>(buf, istride, lstride, tw, sign);
        fft_lines<T, N, P + 1, LINES, THREADS, LF>(buf, istride, lstride, tw, sign);
    }
}

template <typename T, int N> __host__ __device__ constexpr int xy_threads() { return (N >= 96) ? 1024 : (N >= 48 ? 512 : 256); }

// data: [planes][N][N] (y then x); one CTA per plane
template <typename T, int N>
__global__ void __launch_bounds__(xy_threads<T, N>(), (xy_threads<T, N>() <= 512 ? 2 : 1)) k_fft_xy(typename Cplx<T>::t *__restrict__ data,
                                                               const typename Cplx<T>::t *__restrict__ tw, int sign) {
    using C = typename Cplx<T>::t;
    constexpr int THREADS = xy_threads<T, N>();
    constexpr int LD = N + 1;  // padded row
    extern __shared__ __align__(16) unsigned char xy_smem[];
    C *twl = reinterpret_cast<C *>(xy_smem);
    C *buf = twl + N;
    C *g = data + (size_t)blockIdx.x * N * N;
    for (int i = threadIdx.x; i < N; i += THREADS) twl[i] = tw[i];
    for (int i = threadIdx.x; i < N * N; i += THREADS) buf[(i / N) * LD + (i % N)] = g[i];
    __syncthreads();
    fft_lines<T, N, 0, N, THREADS, false>(buf, 1, LD, twl, sign);  // along x: line = y
    fft_lines<T, N, 0, N, THREADS, true>(buf, LD, 1, twl, sign);   // along y: line = x
    for (int i = threadIdx.x; i < N * N; i += THREADS) g[i] = buf[(i / N) * LD + (i % N)];
}

template <typename T, int N> __host__ __device__ constexpr size_t xy_smem_bytes() { return sizeof(typename Cplx<T>::t) * (N + (size_t)N * (N + 1)); }

// Persistent form of k_fft_xy: each CTA walks the planes blockIdx.x, +gridDim.x, ...  A plane
// (N x N contiguous values) arrives by bulk copy into one of two shared-memory buffers while
// the other is transformed, and leaves by bulk store.  Waits are bounded; a wait that runs
// out sets *err and the CTA stops.
//
// FP32, N = 64 (two radix-8 passes per axis): rows are stored 72 values apart (the copies go
// row by row), so that the four rows one warp touches fall on alternate halves of the
// shared-memory banks, and the first x pass writes its outputs 8j + r at 9j + r (an 8 x 9
// padded transpose); with that, every pass reads and writes without bank conflicts.
// Otherwise the plane is one contiguous copy and the x passes take consecutive points of a
// line per thread (y: consecutive lines).
template <typename T, int N> __host__ __device__ constexpr bool xy_padded() { return N == 64 && sizeof(T) == 4; }
template <typename T, int N> __host__ __device__ constexpr int xy_row() { return xy_padded<T, N>() ? 72 : N; }
template <typename T, int N> __host__ __device__ constexpr size_t xy_tma_smem_bytes() {
    return sizeof(typename Cplx<T>::t) * (2 * (size_t)N * xy_row<T, N>() + N);
}
template <typename T, int N> __host__ __device__ constexpr bool xy_tma_fits() { return xy_tma_smem_bytes<T, N>() <= 200 * 1024; }

// The x transforms of a padded 64 x 64 plane (row stride 72): thread t takes butterfly
// j = t % 8 of row t / 8 in both radix-8 passes.  A warp owns its four rows, so only warp
// barriers separate the passes; the caller's block barrier follows.
template <typename T, int THREADS>
__device__ __forceinline__ void fft64_rows_padded(typename Cplx<T>::t *buf, const typename Cplx<T>::t *tw, int sign) {
    using C = typename Cplx<T>::t;
    constexpr int P = 72;
    static_assert(THREADS == 512, "one butterfly of one row per thread");
    const int j = threadIdx.x & 7;
    C *b = buf + (threadIdx.x >> 3) * P;
    C v[8];
    // pass 1 (span 1): inputs j + 8r, outputs 8j + r stored at 9j + r
#pragma unroll
    for (int r = 0; r < 8; ++r) v[r] = b[j + 8 * r];
    dft_small<T, 8>(v, sign);
    __syncwarp();
#pragma unroll
    for (int r = 0; r < 8; ++r) b[9 * j + r] = v[r];
    __syncwarp();
    // pass 2 (span 8): inputs j + 8r (stored at 9r + j) twiddled by w^(jr), outputs j + 8r
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        C x = b[9 * r + j];
        if (r > 0) {
            C w = tw[(j * r) & 63];
            if (sign < 0) w.y = -w.y;
            x = cmul(x, w);
        }
        v[r] = x;
    }
    dft_small<T, 8>(v, sign);
    __syncwarp();
#pragma unroll
    for (int r = 0; r < 8; ++r) b[j + 8 * r] = v[r];
}

// CTAs per SM the register allocator is asked to allow (the padded FP32 planes: three fit in
// shared memory)
template <typename T, int N> __host__ __device__ constexpr int xy_tma_min_blocks() { return xy_padded<T, N>() ? 3 : 1; }

template <typename T, int N>
__global__ void __launch_bounds__(xy_threads<T, N>(), xy_tma_min_blocks<T, N>()) k_fft_xy_tma(typename Cplx<T>::t *__restrict__ data,
                                                                  const typename Cplx<T>::t *__restrict__ tw, int sign,
                                                                  long long nplanes, int *__restrict__ err) {
    using C = typename Cplx<T>::t;
    constexpr int THREADS = xy_threads<T, N>();
    constexpr bool PAD = xy_padded<T, N>();
    constexpr int P = xy_row<T, N>();  // row stride in shared memory
    constexpr uint32_t kPlane = (uint32_t)(sizeof(C) * N * N), kRow = (uint32_t)(sizeof(C) * N);
    extern __shared__ __align__(128) unsigned char xyt_smem[];
    C *buf0 = reinterpret_cast<C *>(xyt_smem);
    C *twl = buf0 + 2 * N * P;
    __shared__ uint64_t full[2];
    __shared__ int abort_flag;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const long long nmine = (long long)blockIdx.x < nplanes ? (nplanes - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    // copy issuers: padded rows, lane 0 of each warp moves its own RW rows in and out (so its
    // wait for its own stores to be read covers the rows it overwrites); else thread 0 moves
    // the whole plane
    constexpr int RW = PAD ? N / (THREADS / 32) : N;
    static_assert(!PAD || N % (THREADS / 32) == 0, "whole rows per warp");
    const bool issuer = PAD ? lane == 0 : tid == 0;
    const int r0 = PAD ? warp * RW : 0;
    auto load_rows = [&](C *dst, const C *src, uint64_t *bar) {
        if constexpr (PAD) {
            for (int r = r0; r < r0 + RW; ++r) bulk_load(dst + r * P, src + r * N, kRow, bar);
        } else {
            bulk_load(dst, src, kPlane, bar);
        }
    };
    auto store_rows = [&](C *dst, const C *src) {
        if constexpr (PAD) {
            for (int r = r0; r < r0 + RW; ++r) bulk_store(dst + r * N, src + r * P, kRow);
        } else {
            bulk_store(dst, src, kPlane);
        }
        bulk_commit();
    };
    if (tid == 0) {
        mbar_init(&full[0], 1);
        mbar_init(&full[1], 1);
        mbar_fence_init();
        abort_flag = 0;
        if (nmine > 0) mbar_arrive_expect_tx(&full[0], kPlane);
    }
    for (int i = tid; i < N; i += THREADS) twl[i] = tw[i];
    __syncthreads();
    if (issuer && nmine > 0) load_rows(buf0, data + (size_t)blockIdx.x * N * N, &full[0]);
    long long i = 0;
    for (; i < nmine; ++i) {
        const int s = (int)(i & 1);
        C *buf = buf0 + s * N * P;
        const long long p = blockIdx.x + i * gridDim.x;
        const bool more = i + 1 < nmine;
        if (!mbar_wait(&full[s], (uint32_t)((i >> 1) & 1))) abort_flag = 1;
        if (tid == 0 && more) mbar_arrive_expect_tx(&full[s ^ 1], kPlane);
        __syncthreads();
        if (abort_flag) break;
        if (issuer && more) {
            bulk_wait_read_all();  // this issuer's stores of the other buffer have been read out
            load_rows(buf0 + (s ^ 1) * N * P, data + (size_t)(p + gridDim.x) * N * N, &full[s ^ 1]);
        }
        if constexpr (PAD) {
            fft64_rows_padded<T, THREADS>(buf, twl, sign);  // along x
            __syncthreads();
        } else {
            fft_lines<T, N, 0, N, THREADS, false>(buf, 1, N, twl, sign);  // along x: line = y
        }
        fft_lines<T, N, 0, N, THREADS, true>(buf, P, 1, twl, sign);  // along y: line = x
        fence_proxy_async_smem();
        __syncthreads();
        if (issuer) store_rows(data + (size_t)p * N * N, buf);
    }
    if (tid == 0 && abort_flag) {
        atomicExch(err, 1);
        // the copy that did not land in time gets one more bounded wait before the CTA exits
        (void)mbar_wait(&full[i & 1], (uint32_t)((i >> 1) & 1));
    }
    if (issuer) bulk_wait_all();
}

template <typename T> __host__ __device__ constexpr int z_tl() { return sizeof(T) == 8 ? 16 : 32; }

// data: [planes][nz = N][ny][nx]; CTA = (plane, y, x-tile of TL)
template <typename T, int N>
__global__ void __launch_bounds__(256) k_fft_z(typename Cplx<T>::t *__restrict__ data, const typename Cplx<T>::t *__restrict__ tw,
                                              int nx, int ny, int sign) {
    using C = typename Cplx<T>::t;
    constexpr int TL = z_tl<T>();
    constexpr int LD = TL + 1;
    extern __shared__ __align__(16) unsigned char z_smem[];
    C *twl = reinterpret_cast<C *>(z_smem);
    C *buf = twl + N;
    const int xt = nx / TL;
    const long long t = blockIdx.x;
    const int ix0 = (int)(t % xt) * TL;
    const long long rest = t / xt;  // plane * ny + iy
    const long long p = rest / ny, iy = rest % ny;
    const long long plane = (long long)nx * ny * N;
    C *g = data + p * plane + iy * nx + ix0;
    const long long zs = (long long)nx * ny;
    for (int i = threadIdx.x; i < N; i += 256) twl[i] = tw[i];
    {
        // all loads of the column tile in flight before the first shared-memory store
        constexpr int PER = (N * TL + 255) / 256;
        C t[PER];
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            const int f = threadIdx.x + 256 * k;
            if ((N * TL) % 256 == 0 || f < N * TL) t[k] = g[(f / TL) * zs + f % TL];
        }
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            const int f = threadIdx.x + 256 * k;
            if ((N * TL) % 256 == 0 || f < N * TL) buf[(f / TL) * LD + f % TL] = t[k];
        }
    }
    __syncthreads();
    fft_lines<T, N, 0, TL, 256, true>(buf, LD, 1, twl, sign);
    for (int f = threadIdx.x; f < N * TL; f += 256) {
        const int i = f / TL, l = f % TL;
        g[i * zs + l] = buf[i * LD + l];
    }
}

template <typename T, int N> __host__ __device__ constexpr size_t z_smem_bytes() { return sizeof(typename Cplx<T>::t) * (N + (size_t)N * (z_tl<T>() + 1)); }

}  // namespace mdft
