// Kernels of the warm-start network: periodic 3-D convolutions as gather-GEMMs on FP32
// CUDA cores (BF16 weights, FP32 activations and accumulation), GELU, bias and loss
// reductions, Adam.
//
// Layouts.  A volume of C channels on a d x h x w grid is [C][z][y][x] with x fastest,
// the point order of the solver's xi(no, nx, ny, nz) with io dropped.  Weights of a
// convolution are [cout][cin][kz][ky][kx]; weights of the transposed (up-sampling)
// convolution are [cin][cout][kz][ky][kx] (the coarse channel first).
//
// Three convolution kinds, all periodic like the solver's box:
//   KS=3, S=1: 3x3x3, wrap-around padding of one voxel;
//   KS=2, S=2: 2x2x2 stride 2 (down-sampling), and its transpose (up-sampling);
//   KS=1, S=1: pointwise (the output head).
// Every convolution and both of its gradients is one tile kernel, k_conv_gemm<MODE,...>:
// a 64-voxel x 32-channel output tile per CTA, reduction chunks of 32 staged in shared
// memory (A gathered from the activation volume, B from the weights, converted to FP32).
#pragma once

#include <cuda_bf16.h>

#include "common.cuh"

namespace mdft {
namespace wn {

struct Vol {
    int d, h, w;
    __host__ __device__ long long n() const { return (long long)d * h * w; }
};

constexpr int kBM = 64;   // voxels per tile
constexpr int kBN = 32;   // channels per tile
constexpr int kBK = 32;   // reduction chunk
constexpr int kThreads = 256;

enum ConvMode {
    kFwd = 0,     // Y[co][o] = sum_{ci,k} W[co][ci][k] X[ci][o*S - P + k]           (conv forward)
    kBwdData = 1, // dX[ci][i] = sum_{co,k} W[co][ci][k] dY[co][i + P - k]          (S = 1 only)
    kParity = 2,  // F[cf][2o+a] = sum_cc W[cc][cf][a] C[cc][o]                      (KS = 2, S = 2:
                  //  the transposed convolution, and the data gradient of the stride-2 conv)
};

struct ConvArgs {
    const float *x;            // gathered operand (kFwd: input X; kBwdData: dY; kParity: coarse C)
    const __nv_bfloat16 *wt;   // weights
    const float *bias;         // per output channel, or null
    float *y;                  // output volume
    int cin, cout;             // channels of the gathered operand / of the output
    Vol vin, vout;             // grid of the gathered operand / of the output
    int accumulate;            // 1: y += result, 0: y = result
};

__device__ __forceinline__ int wrapi(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

// One output tile.  blockIdx.x: voxel tile, blockIdx.y: channel tile, blockIdx.z: parity
// class a = (az*2 + ay)*2 + ax (kParity only).
template <int MODE, int KS, int S>
__global__ void __launch_bounds__(kThreads) k_conv_gemm(ConvArgs a) {
    constexpr int K3 = KS * KS * KS;
    constexpr int P = KS == 3 ? 1 : 0;
    __shared__ float As[kBK][kBM];
    __shared__ __align__(16) float Bs[kBK][kBN + 4];
    const int tid = threadIdx.x;
    const int v = tid & (kBM - 1);     // this thread's voxel in the tile
    const int cg = tid >> 6;           // its group of 8 output channels
    const int co0 = blockIdx.y * kBN;
    const int par = MODE == kParity ? (int)blockIdx.z : 0;
    // voxels are enumerated over the grid the reduction is gathered on: the output grid
    // for kFwd / kBwdData, the coarse grid for kParity
    const Vol vg = MODE == kParity ? a.vin : a.vout;
    const long long nv = vg.n();
    const long long o = (long long)blockIdx.x * kBM + v;
    const bool live = o < nv;
    int ox = 0, oy = 0, oz = 0;
    if (live) {
        ox = (int)(o % vg.w);
        long long t = o / vg.w;
        oy = (int)(t % vg.h);
        oz = (int)(t / vg.h);
    }
    // reduction length: kFwd cin*K3, kBwdData cin*K3 (cin = channels of dY), kParity cin
    const int Ktot = MODE == kParity ? a.cin : a.cin * K3;
    const long long nin = a.vin.n();
    float acc[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[j] = 0.f;
    for (int k0 = 0; k0 < Ktot; k0 += kBK) {
        // A: this thread's voxel, reduction rows (tid >> 6) + 4 j
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int kr = cg + 4 * j;
            const int kk = k0 + kr;
            float val = 0.f;
            if (live && kk < Ktot) {
                if (MODE == kParity) {
                    val = a.x[(long long)kk * nin + o];
                } else {
                    const int c = kk / K3, kof = kk - c * K3;
                    const int kx = kof % KS, ky = (kof / KS) % KS, kz = kof / (KS * KS);
                    int ix, iy, iz;
                    if (MODE == kFwd) {
                        ix = ox * S - P + kx; iy = oy * S - P + ky; iz = oz * S - P + kz;
                    } else {
                        ix = ox + P - kx; iy = oy + P - ky; iz = oz + P - kz;
                    }
                    if (P) { ix = wrapi(ix, a.vin.w); iy = wrapi(iy, a.vin.h); iz = wrapi(iz, a.vin.d); }
                    val = a.x[(long long)c * nin + ((long long)iz * a.vin.h + iy) * a.vin.w + ix];
                }
            }
            As[kr][v] = val;
        }
        // B: rows of the weights, (channel c, reduction kk) -> Bs[kk][c]
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int e = tid + kThreads * j;
            const int c = e >> 5, kr = e & 31;
            const int co = co0 + c, kk = k0 + kr;
            float val = 0.f;
            if (co < a.cout && kk < Ktot) {
                long long wi;
                if (MODE == kFwd) {
                    wi = (long long)co * Ktot + kk;                           // W[co][ci][k]
                } else if (MODE == kBwdData) {
                    const int cc = kk / K3, kof = kk - cc * K3;               // W[cc][co][k]
                    wi = ((long long)cc * a.cout + co) * K3 + kof;
                } else {
                    wi = ((long long)kk * a.cout + co) * 8 + par;             // W[kk][co][a]
                }
                val = __bfloat162float(a.wt[wi]);
            }
            Bs[kr][c] = val;
        }
        __syncthreads();
#pragma unroll 8
        for (int k = 0; k < kBK; ++k) {
            const float av = As[k][v];
            const float4 b0 = *reinterpret_cast<const float4 *>(&Bs[k][cg * 8]);
            const float4 b1 = *reinterpret_cast<const float4 *>(&Bs[k][cg * 8 + 4]);
            acc[0] = fmaf(av, b0.x, acc[0]); acc[1] = fmaf(av, b0.y, acc[1]);
            acc[2] = fmaf(av, b0.z, acc[2]); acc[3] = fmaf(av, b0.w, acc[3]);
            acc[4] = fmaf(av, b1.x, acc[4]); acc[5] = fmaf(av, b1.y, acc[5]);
            acc[6] = fmaf(av, b1.z, acc[6]); acc[7] = fmaf(av, b1.w, acc[7]);
        }
        __syncthreads();
    }
    if (!live) return;
    long long oi = o;
    if (MODE == kParity) {
        const int ax = par & 1, ay = (par >> 1) & 1, az = par >> 2;
        oi = ((long long)(2 * oz + az) * a.vout.h + (2 * oy + ay)) * a.vout.w + (2 * ox + ax);
    }
    const long long nout = a.vout.n();
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int co = co0 + cg * 8 + j;
        if (co >= a.cout) break;
        float r = acc[j];
        if (a.bias) r += a.bias[co];
        float *dst = a.y + (long long)co * nout + oi;
        *dst = a.accumulate ? *dst + r : r;
    }
}

struct WgradArgs {
    const float *dy;   // [cout][nout]: gradient at the conv output (coarse for KS=2)
    const float *x;    // [cin][nin]: the conv input
    float *part;       // [nsplit][cout][cin*K3]
    int cin, cout;
    Vol vin, vout;
    long long per_split;  // output voxels per split (a multiple of kBK)
};

// dW[co][ci][k] = sum_o dY[co][o] X[ci][o*S - P + k]: a 32-channel x 64-column tile per CTA
// over one split of the output voxels (blockIdx.z), partial sums to part[split].
template <int KS, int S>
__global__ void __launch_bounds__(kThreads) k_conv_wgrad(WgradArgs a) {
    constexpr int K3 = KS * KS * KS;
    constexpr int P = KS == 3 ? 1 : 0;
    __shared__ __align__(16) float As[kBK][kBN + 4];  // [voxel][co]
    __shared__ float Bs[kBK][kBM];                    // [voxel][column]
    const int tid = threadIdx.x;
    const int col = tid & (kBM - 1);
    const int cg = tid >> 6;
    const int Ktot = a.cin * K3;
    const int kk = blockIdx.x * kBM + col;  // this thread's weight column
    const bool colok = kk < Ktot;
    int ci = 0, kx = 0, ky = 0, kz = 0;
    if (colok) {
        ci = kk / K3;
        const int kof = kk - ci * K3;
        kx = kof % KS; ky = (kof / KS) % KS; kz = kof / (KS * KS);
    }
    const int co0 = blockIdx.y * kBN;
    const long long nout = a.vout.n(), nin = a.vin.n();
    const long long s0 = (long long)blockIdx.z * a.per_split;
    const long long s1 = s0 + a.per_split < nout ? s0 + a.per_split : nout;
    float acc[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[j] = 0.f;
    for (long long o0 = s0; o0 < s1; o0 += kBK) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {  // dY rows: (co, voxel) -> As[voxel][co]
            const int e = tid + kThreads * j;
            const int c = e >> 5, vv = e & 31;
            const long long o = o0 + vv;
            const int co = co0 + c;
            As[vv][c] = (co < a.cout && o < s1) ? a.dy[(long long)co * nout + o] : 0.f;
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) {  // X gathered at this column's offset
            const int vv = cg + 4 * j;
            const long long o = o0 + vv;
            float val = 0.f;
            if (colok && o < s1) {
                const int ox = (int)(o % a.vout.w);
                const long long t = o / a.vout.w;
                const int oy = (int)(t % a.vout.h), oz = (int)(t / a.vout.h);
                int ix = ox * S - P + kx, iy = oy * S - P + ky, iz = oz * S - P + kz;
                if (P) { ix = wrapi(ix, a.vin.w); iy = wrapi(iy, a.vin.h); iz = wrapi(iz, a.vin.d); }
                val = a.x[(long long)ci * nin + ((long long)iz * a.vin.h + iy) * a.vin.w + ix];
            }
            Bs[vv][col] = val;
        }
        __syncthreads();
#pragma unroll 8
        for (int k = 0; k < kBK; ++k) {
            const float bv = Bs[k][col];
            const float4 a0 = *reinterpret_cast<const float4 *>(&As[k][cg * 8]);
            const float4 a1 = *reinterpret_cast<const float4 *>(&As[k][cg * 8 + 4]);
            acc[0] = fmaf(a0.x, bv, acc[0]); acc[1] = fmaf(a0.y, bv, acc[1]);
            acc[2] = fmaf(a0.z, bv, acc[2]); acc[3] = fmaf(a0.w, bv, acc[3]);
            acc[4] = fmaf(a1.x, bv, acc[4]); acc[5] = fmaf(a1.y, bv, acc[5]);
            acc[6] = fmaf(a1.z, bv, acc[6]); acc[7] = fmaf(a1.w, bv, acc[7]);
        }
        __syncthreads();
    }
    if (!colok) return;
    float *dst = a.part + (long long)blockIdx.z * a.cout * Ktot;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int co = co0 + cg * 8 + j;
        if (co >= a.cout) break;
        dst[(long long)co * Ktot + kk] = acc[j];
    }
}

// g[i] (+)= sum over splits of part[s][i], in split order
__global__ void k_wgrad_reduce(const float *__restrict__ part, float *__restrict__ g, int nsplit, long long n, int accumulate) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        float s = 0.f;
        for (int k = 0; k < nsplit; ++k) s += part[(long long)k * n + i];
        g[i] = accumulate ? g[i] + s : s;
    }
}

__device__ __forceinline__ float gelu_f(float z) { return 0.5f * z * (1.f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z) {
    return 0.5f * (1.f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

// a = GELU(z) (erf form)
__global__ void k_gelu(const float *__restrict__ z, float *__restrict__ out, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = gelu_f(z[i]);
}

// g *= GELU'(z)
__global__ void k_gelu_bwd(const float *__restrict__ z, float *__restrict__ g, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        g[i] *= gelu_grad(z[i]);
}

// y += x
__global__ void k_add(float *__restrict__ y, const float *__restrict__ x, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        y[i] += x[i];
}

// db[c] (+)= sum_v g[c][v]; one block per channel, FP64 partials in a fixed order
__global__ void __launch_bounds__(256) k_bias_grad(const float *__restrict__ g, float *__restrict__ db, long long nv, int accumulate) {
    __shared__ double red[256];
    const int c = blockIdx.x;
    const float *p = g + (long long)c * nv;
    double s = 0.0;
    for (long long i = threadIdx.x; i < nv; i += 256) s += p[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) db[c] = accumulate ? db[c] + (float)red[0] : (float)red[0];
}

// masked squared error over C channels: loss = sum_v m_v sum_c (y - t)^2 * inv_norm,
// g = dloss/dy; per-block FP64 partials to part[blockIdx.x]
__global__ void __launch_bounds__(256) k_mse(const float *__restrict__ y, const float *__restrict__ t, const float *__restrict__ mask,
                                             float *__restrict__ g, double *__restrict__ part, int C, long long nv, float inv_norm) {
    __shared__ double red[256];
    double s = 0.0;
    for (long long v = blockIdx.x * 256LL + threadIdx.x; v < nv; v += (long long)gridDim.x * 256) {
        const float m = mask ? mask[v] : 1.f;
        for (int c = 0; c < C; ++c) {
            const float d = y[(long long)c * nv + v] - t[(long long)c * nv + v];
            g[(long long)c * nv + v] = 2.f * m * d * inv_norm;
            s += (double)(m * d * d);
        }
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0] * (double)inv_norm;
}

// acc[0] += sum of the first n partials (one thread block)
__global__ void k_sum_into(const double *__restrict__ part, int n, double *__restrict__ acc) {
    __shared__ double red[256];
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += 256) s += part[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) acc[0] += red[0];
}

// Adam (Kingma & Ba 2015) on the FP32 master parameters; the BF16 copy used by the
// kernels is rewritten.  gscale multiplies the accumulated gradient (1/batch).
__global__ void k_adam(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m, float *__restrict__ v,
                       __nv_bfloat16 *__restrict__ pb, long long n, float lr, float b1, float b2, float eps, float c1, float c2,
                       float gscale) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i] * gscale;
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float pi = p[i] - lr * (mi * c1) / (sqrtf(vi * c2) + eps);
        p[i] = pi;
        pb[i] = __float2bfloat16_rn(pi);
    }
}

__global__ void k_to_bf16(const float *__restrict__ p, __nv_bfloat16 *__restrict__ pb, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        pb[i] = __float2bfloat16_rn(p[i]);
}

}  // namespace wn
}  // namespace mdft
