// Rotated OZ step for FP32 evaluations (S3-S5 of src/module_energy_cproj_mrso.f90:441-674,
// same arithmetic as k_oz2<float>), one thread per (q, -q) pair.
//
// Every index of the step -- projection positions, rotation-matrix entries, the terms of the
// two rotations and of the OZ sums -- is a compile-time function of (MMAX, MRSO), so with the
// loops unrolled the rotation matrices live in registers and the projections in a per-thread
// shared-memory slice addressed with immediates.  Only the independent half of each level
// of R(q) is computed and kept (the recursion's dest entries); the filled half is derived on
// use as (s Re, -s Im), s = (-1)^(m+m1), as the reference's symmetric fill stores it.
//
// Neighbouring threads take neighbouring k-points of one (iz) plane, so the loads of q and
// of its partner -q from the projection planes are coalesced without staging.  The first
// c(k) coefficient of each output (ia0) and the recursion coefficients come in as kernel
// parameters (uniform across the warp).
#pragma once

#include "common.cuh"
#include "k_fft.cuh"
#include "k_oz.cuh"
#include "k_oz2.cuh"

namespace mdft {

constexpr int kOzpThreads = 128;
#ifndef MDFT_OZP_MIN_BLOCKS
#define MDFT_OZP_MIN_BLOCKS 1
#endif
constexpr int kOzpMinBlocks = MDFT_OZP_MIN_BLOCKS;  // resident CTAs asked of the register allocator
#ifndef MDFT_OZD_MIN_BLOCKS
#define MDFT_OZD_MIN_BLOCKS 2
#endif
constexpr int kOzdMinBlocks = MDFT_OZD_MIN_BLOCKS;
constexpr int kOzpMaxNp = 64;
constexpr int kOzpMaxRec = 48;

struct OzpParams {
    int ia0[kOzpMaxNp];        // first c coefficient of each output's OZ sum
    float rc[3 * kOzpMaxRec];  // recursion coefficients, three per computed entry
};

template <int MM, int MR> struct OzShape {
    __host__ __device__ static constexpr int np() {
        int s = 0;
        for (int m = 0; m <= MM; ++m) s += (2 * m + 1) * (m / MR + 1);
        return s;
    }
    __host__ __device__ static constexpr int pidx(int m, int mup, int mu2) {
        int off = 0;
        for (int k = 0; k < m; ++k) off += (2 * k + 1) * (k / MR + 1);
        return off + (mup + m) * (m / MR + 1) + mu2;
    }
    __host__ __device__ static constexpr int m1min(int m) { return m > 0 ? 1 : 0; }
    __host__ __device__ static constexpr int level_count(int l) {
        int c = 0;
        for (int m = -l; m <= l; ++m) c += l - m1min(m) + 1;
        return c;
    }
    // position of the computed entry (l, m, m1), l >= 2, among all computed entries
    __host__ __device__ static constexpr int hidx(int l, int m, int m1) {
        int off = 0;
        for (int k = 2; k < l; ++k) off += level_count(k);
        for (int mm = -l; mm < m; ++mm) off += l - m1min(mm) + 1;
        return off + (m1 - m1min(m));
    }
    __host__ __device__ static constexpr int nhalf() {
        int c = 0;
        for (int l = 2; l <= MM; ++l) c += level_count(l);
        return c;
    }
};

template <int MM, int MR, int NH>
__device__ __forceinline__ float2 ozp_rget(const float2 (&R1)[9], const float2 (&Rh)[NH], int l, int m, int m1) {
    using S = OzShape<MM, MR>;
    if (l == 0) return make_float2(1.f, 0.f);
    if (l == 1) return R1[(m + 1) * 3 + (m1 + 1)];
    if (m1 >= S::m1min(m)) return Rh[S::hidx(l, m, m1)];
    const float2 v = Rh[S::hidx(l, -m, -m1)];
    const float s = ((m + m1) & 1) ? -1.f : 1.f;
    return make_float2(s * v.x, -s * v.y);
}

__device__ __forceinline__ void ozp_fma(float2 &acc, float2 a, float2 b) {  // acc += a*b
    acc.x += a.x * b.x - a.y * b.y;
    acc.y += a.x * b.y + a.y * b.x;
}
__device__ __forceinline__ void ozp_fmac(float2 &acc, float2 a, float2 b) {  // acc += a*conj(b)
    acc.x += a.x * b.x + a.y * b.y;
    acc.y += a.y * b.x - a.x * b.y;
}

template <int MM, int MR>
__global__ void __launch_bounds__(kOzpThreads, kOzpMinBlocks) k_ozp(float2 *__restrict__ planes, const float2 *__restrict__ ctab, Oz2Args a,
                                                     OzpParams pp, const float2 *__restrict__ cq) {
    using S = OzShape<MM, MR>;
    constexpr int NP = S::np();
    constexpr int NH = S::nhalf() > 0 ? S::nhalf() : 1;
    constexpr int B = kOzpThreads;
    extern __shared__ __align__(16) float2 ozp_smem[];  // [2 NP][B]: q side, then -q side
    const int t = threadIdx.x;
    float2 *sq = ozp_smem + t;            // element ip of the q side: sq[ip * B]
    float2 *smq = ozp_smem + NP * B + t;  // element ip of the -q side
    const long long kk = (long long)blockIdx.x * B + t;
    if (kk >= a.nk) return;
    const int ix = (int)(kk % a.nx), iy = (int)((kk / a.nx) % a.ny), iz = (int)(kk / ((long long)a.nx * a.ny));
    const int ixm = (a.nx - ix) % a.nx, iym = (a.ny - iy) % a.ny, izm = (a.nz - iz) % a.nz;
    if ((iz == 0 || 2 * iz == a.nz) && (long long)iy * a.nx + ix > (long long)iym * a.nx + ixm) return;  // partner is the q
    const bool selfconj = ix == ixm && iy == iym && iz == izm;
    const bool nyq = (2 * ix == a.nx) || (2 * iy == a.ny) || (2 * iz == a.nz);
    const long long kq = ((long long)iz * a.ny + iy) * a.nx + ix;
    const long long km = ((long long)izm * a.ny + iym) * a.nx + ixm;

    const double qx = (ix <= a.nx / 2 ? ix : ix - a.nx) * a.twopi_lx;
    const double qy = (iy <= a.ny / 2 ? iy : iy - a.ny) * a.twopi_ly;
    const double qz = (iz <= a.nz / 2 ? iz : iz - a.nz) * a.twopi_lz;

    // ---- R(q): l = 1 block, then the recursion of src/module_rotation.f90:119-247 ----
    float2 R1[9];
    float2 Rh[NH];
    {
        float r3[3], r2[3], r1[3];
        if (qx == 0.0 && qy == 0.0 && qz == 0.0) { r3[0] = 0; r3[1] = 0; r3[2] = 1; }
        else { r3[0] = (float)qx; r3[1] = (float)qy; r3[2] = (float)qz; }
        if (r3[0] != 0.f || r3[1] != 0.f) { r2[0] = -r3[1]; r2[1] = r3[0]; r2[2] = 0; }
        else { r2[0] = 0; r2[1] = r3[2]; r2[2] = -r3[1]; }
        const float n3 = sqrtf(r3[0] * r3[0] + r3[1] * r3[1] + r3[2] * r3[2]);
        const float n2 = sqrtf(r2[0] * r2[0] + r2[1] * r2[1] + r2[2] * r2[2]);
#pragma unroll
        for (int i = 0; i < 3; ++i) { r3[i] /= n3; r2[i] /= n2; }
        r1[0] = r2[1] * r3[2] - r2[2] * r3[1];
        r1[1] = r2[2] * r3[0] - r2[0] * r3[2];
        r1[2] = r2[0] * r3[1] - r2[1] * r3[0];
        const float sqrt2 = 1.4142135623730950488016887242097f;
        R1[0] = make_float2((r2[1] + r1[0]) * 0.5f, (r1[1] - r2[0]) * 0.5f);   // (-1,-1)
        R1[1] = make_float2(r3[0] / sqrt2, r3[1] / sqrt2);                    // (-1, 0)
        R1[2] = make_float2((r2[1] - r1[0]) * 0.5f, (-r1[1] - r2[0]) * 0.5f);  // (-1, 1)
        R1[3] = make_float2(r1[2] / sqrt2, -r2[2] / sqrt2);                   // ( 0,-1)
        R1[4] = make_float2(r3[2], 0.f);                                      // ( 0, 0)
        R1[5] = make_float2(-r1[2] / sqrt2, -r2[2] / sqrt2);                  // ( 0, 1)
        R1[6] = make_float2((r2[1] - r1[0]) * 0.5f, (r1[1] + r2[0]) * 0.5f);   // ( 1,-1)
        R1[7] = make_float2(-r3[0] / sqrt2, r3[1] / sqrt2);                   // ( 1, 0)
        R1[8] = make_float2((r2[1] + r1[0]) * 0.5f, (r2[0] - r1[1]) * 0.5f);   // ( 1, 1)
    }
    if constexpr (MM >= 1) {
#pragma unroll
        for (int l = 2; l <= MM; ++l) {
#pragma unroll
            for (int m = -l; m <= l; ++m) {
#pragma unroll
                for (int m1 = S::m1min(m); m1 <= l; ++m1) {
                    const int e = S::hidx(l, m, m1);
                    const int l1 = l - 1;
                    // terms t = 0..2: coefficient, level-1 entry X, level l-1 entry U
                    float2 val = make_float2(0.f, 0.f);
                    auto term = [&](int tt, int xm, int xm1, int um, int um1) {
                        if (um < -l1 || um > l1 || um1 < -l1 || um1 > l1) return;
                        const float2 X = R1[(xm + 1) * 3 + (xm1 + 1)];
                        const float2 U = ozp_rget<MM, MR, NH>(R1, Rh, l1, um, um1);
                        const float cf = pp.rc[3 * e + tt];
                        val.x += cf * (X.x * U.x - X.y * U.y);
                        val.y += cf * (X.x * U.y + X.y * U.x);
                    };
                    if (m1 < l) {
                        if (m == -l) term(0, -1, 0, m + 1, m1);
                        else if (m == l) term(0, 1, 0, m - 1, m1);
                        else { term(0, 0, 0, m, m1); term(1, 1, 0, m - 1, m1); term(2, -1, 0, m + 1, m1); }
                    } else {
                        if (m == -l) term(0, -1, 1, m + 1, m1 - 1);
                        else if (m == l) term(0, 1, 1, m - 1, m1 - 1);
                        else { term(0, 0, 1, m, m1 - 1); term(1, 1, 1, m - 1, m1 - 1); term(2, -1, 1, m + 1, m1 - 1); }
                    }
                    Rh[e] = (m == 0 && m1 == 0) ? make_float2(val.x, -val.y) : val;
                }
            }
        }
        // flush |Re|, |Im| < epsilon(1.) (:491-492); the filled half follows its source
        auto flush = [](float2 &v) {
            if (fabsf(v.x) < (float)kEpsSp) v.x = 0.f;
            if (fabsf(v.y) < (float)kEpsSp) v.y = 0.f;
        };
#pragma unroll
        for (int i = 0; i < 9; ++i) flush(R1[i]);
#pragma unroll
        for (int i = 0; i < NH; ++i) flush(Rh[i]);
    }

    // ---- forward rotation (:505-523), block (m, mu2) at a time, into shared memory ----
#pragma unroll
    for (int m = 0; m <= MM; ++m)
#pragma unroll
        for (int mu2 = 0; mu2 <= m / MR; ++mu2) {
            float2 dq[2 * MM + 1], dmq[2 * MM + 1];
#pragma unroll
            for (int mup = -m; mup <= m; ++mup) {
                const size_t off = (size_t)S::pidx(m, mup, mu2) * a.N;
                dq[mup + m] = planes[off + kq];
                dmq[mup + m] = planes[off + km];
            }
            const float sg = (m & 1) ? -1.f : 1.f;
#pragma unroll
            for (int khi = -m; khi <= m; ++khi) {
                float2 s = make_float2(0.f, 0.f), u = make_float2(0.f, 0.f);
#pragma unroll
                for (int mup = -m; mup <= m; ++mup) {
                    ozp_fma(s, dq[mup + m], ozp_rget<MM, MR, NH>(R1, Rh, m, mup, khi));
                    ozp_fma(u, dmq[mup + m], ozp_rget<MM, MR, NH>(R1, Rh, m, mup, -khi));
                }
                const int o = S::pidx(m, khi, mu2);
                sq[o * B] = s;
                smq[o * B] = make_float2(sg * u.x, sg * u.y);
            }
        }

    // ---- interpolated c (:534-539) and the OZ sums (:561-606), one chi block at a time ----
    // cq (cubic grid in a cubic box): c already interpolated at every |q|^2 = (2 pi/L)^2 s2 of
    // the grid, row s2; otherwise the two bracketing rows of the table and their weight
    const double nrm = sqrt(qx * qx + qy * qy + qz * qz);
    const double eff = nrm / a.dq + 1.0;
    const int iq = (int)eff;
    const float alpha = (float)(eff - iq);
    const float2 *c0 = ctab + (size_t)(iq - 1) * a.ncoef;
    const float2 *c1 = ctab + (size_t)iq * a.ncoef;
    const float2 *crow = nullptr;
    if (cq) {
        const int sx = ix <= a.nx / 2 ? ix : ix - a.nx, sy = iy <= a.ny / 2 ? iy : iy - a.ny, sz = iz <= a.nz / 2 ? iz : iz - a.nz;
        crow = cq + (size_t)(sx * sx + sy * sy + sz * sz) * a.ncoef;
    }
#pragma unroll
    for (int khi = -MM; khi <= MM; ++khi) {
        constexpr int BMAX = 2 * (MM / MR + 1) * (MM + 1);
        float2 gs[BMAX], gm[BMAX];
        int nb = 0;
#pragma unroll
        for (int m = (khi < 0 ? -khi : khi); m <= MM; ++m)
#pragma unroll
            for (int mu2 = 0; mu2 <= m / MR; ++mu2) {
                const int ip = S::pidx(m, khi, mu2);
                float2 s = make_float2(0.f, 0.f), u = make_float2(0.f, 0.f);
                int k = 0;
#pragma unroll
                for (int n = (khi < 0 ? -khi : khi); n <= MM; ++n)
#pragma unroll
                    for (int nu2 = -n / MR; nu2 <= n / MR; ++nu2, ++k) {
                        const int ia = pp.ia0[ip] + k;
                        float2 ce;
                        if (crow) {
                            ce = crow[ia];
                        } else {
                            const float2 A0 = c0[ia], A1 = c1[ia];
                            ce.x = alpha * A1.x + (1.f - alpha) * A0.x;
                            ce.y = alpha * A1.y + (1.f - alpha) * A0.y;
                        }
                        const int jp = S::pidx(n, khi, nu2 < 0 ? -nu2 : nu2);
                        if (nu2 < 0) {
                            ozp_fma(s, ce, sq[jp * B]);
                            ozp_fma(u, ce, smq[jp * B]);
                        } else {
                            ozp_fmac(s, ce, smq[jp * B]);
                            ozp_fmac(u, ce, sq[jp * B]);
                        }
                    }
                gs[nb] = s;
                gm[nb] = u;
                ++nb;
            }
        // the block's inputs are no longer needed: write gamma in place
        nb = 0;
#pragma unroll
        for (int m = (khi < 0 ? -khi : khi); m <= MM; ++m)
#pragma unroll
            for (int mu2 = 0; mu2 <= m / MR; ++mu2) {
                const int ip = S::pidx(m, khi, mu2);
                sq[ip * B] = gs[nb];
                smq[ip * B] = gm[nb];
                ++nb;
            }
    }

    // ---- back rotation with conj(R) (:611-641), straight to the planes ----
#pragma unroll
    for (int m = 0; m <= MM; ++m)
#pragma unroll
        for (int mu2 = 0; mu2 <= m / MR; ++mu2) {
            float2 g[2 * MM + 1], gmv[2 * MM + 1];
#pragma unroll
            for (int k = -m; k <= m; ++k) {
                g[k + m] = sq[S::pidx(m, k, mu2) * B];
                gmv[k + m] = smq[S::pidx(m, k, mu2) * B];
            }
            const float sg = (m & 1) ? -1.f : 1.f;
#pragma unroll
            for (int khi = -m; khi <= m; ++khi) {  // output (m, mup = khi, mu2)
                float2 s = make_float2(0.f, 0.f), u = make_float2(0.f, 0.f);
#pragma unroll
                for (int k = -m; k <= m; ++k) {
                    ozp_fmac(s, g[k + m], ozp_rget<MM, MR, NH>(R1, Rh, m, khi, k));
                    ozp_fmac(u, gmv[k + m], ozp_rget<MM, MR, NH>(R1, Rh, m, khi, -k));
                }
                u.x *= sg;
                u.y *= sg;
                if (selfconj && nyq) u.y = -u.y;
                const size_t off = (size_t)S::pidx(m, khi, mu2) * a.N;
                if (!selfconj) planes[off + kq] = s;
                planes[off + km] = u;
            }
        }
}

// The same step with the rotation matrices factored: R^m_{mu' chi}(q) = e^{-i mu' alpha}
// D^m_{mu' chi}, alpha the azimuth of q (0 when q is along z) and D real -- the recursion of
// src/module_rotation.f90:119-247 pairs indices as m = x + u in every term, so the phases
// factor out of it and D follows the same recursion in real arithmetic from
// D^1(x, x1) = Re(R^1(x, x1) e^{i x alpha}).  A rotation then costs a phase per input and two
// FMAs per term instead of four, and D takes half the registers of R.  The reference's
// flush of R's parts below epsilon(1.) (:491-492) is not reproduced (FP32 evaluations
// only; its effect is below FP32 rounding of the sums).
template <int MM, int MR, int NH>
__device__ __forceinline__ float ozd_dget(const float (&D1)[9], const float (&Dh)[NH], int l, int m, int m1) {
    using S = OzShape<MM, MR>;
    if (l == 0) return 1.f;
    if (l == 1) return D1[(m + 1) * 3 + (m1 + 1)];
    if (m1 >= S::m1min(m)) return Dh[S::hidx(l, m, m1)];
    const float s = ((m + m1) & 1) ? -1.f : 1.f;
    return s * Dh[S::hidx(l, -m, -m1)];
}

template <int MM, int MR>
__global__ void __launch_bounds__(kOzpThreads, kOzdMinBlocks) k_ozd(float2 *__restrict__ planes, const float2 *__restrict__ ctab, Oz2Args a,
                                                     OzpParams pp, const float2 *__restrict__ cq) {
    using S = OzShape<MM, MR>;
    constexpr int NP = S::np();
    constexpr int NH = S::nhalf() > 0 ? S::nhalf() : 1;
    constexpr int B = kOzpThreads;
    extern __shared__ __align__(16) float2 ozp_smem[];  // [2 NP][B]: q side, then -q side
    const int t = threadIdx.x;
    float2 *sq = ozp_smem + t;
    float2 *smq = ozp_smem + NP * B + t;
    const long long kk = (long long)blockIdx.x * B + t;
    if (kk >= a.nk) return;
    const int ix = (int)(kk % a.nx), iy = (int)((kk / a.nx) % a.ny), iz = (int)(kk / ((long long)a.nx * a.ny));
    const int ixm = (a.nx - ix) % a.nx, iym = (a.ny - iy) % a.ny, izm = (a.nz - iz) % a.nz;
    if ((iz == 0 || 2 * iz == a.nz) && (long long)iy * a.nx + ix > (long long)iym * a.nx + ixm) return;  // partner is the q
    const bool selfconj = ix == ixm && iy == iym && iz == izm;
    const bool nyq = (2 * ix == a.nx) || (2 * iy == a.ny) || (2 * iz == a.nz);
    const long long kq = ((long long)iz * a.ny + iy) * a.nx + ix;
    const long long km = ((long long)izm * a.ny + iym) * a.nx + ixm;

    const double qx = (ix <= a.nx / 2 ? ix : ix - a.nx) * a.twopi_lx;
    const double qy = (iy <= a.ny / 2 ? iy : iy - a.ny) * a.twopi_ly;
    const double qz = (iz <= a.nz / 2 ? iz : iz - a.nz) * a.twopi_lz;

    // ---- the l = 1 block of the q frame (as k_ozp), then D^1 = Re(R^1 e^{i x alpha}) ----
    float D1[9];
    float2 ph[MM + 1];  // e^{-i mu alpha}, mu = 0..MM (negative mu: the conjugates)
    {
        float r3[3], r2[3], r1[3];
        if (qx == 0.0 && qy == 0.0 && qz == 0.0) { r3[0] = 0; r3[1] = 0; r3[2] = 1; }
        else { r3[0] = (float)qx; r3[1] = (float)qy; r3[2] = (float)qz; }
        if (r3[0] != 0.f || r3[1] != 0.f) { r2[0] = -r3[1]; r2[1] = r3[0]; r2[2] = 0; }
        else { r2[0] = 0; r2[1] = r3[2]; r2[2] = -r3[1]; }
        const float n3 = sqrtf(r3[0] * r3[0] + r3[1] * r3[1] + r3[2] * r3[2]);
        const float n2 = sqrtf(r2[0] * r2[0] + r2[1] * r2[1] + r2[2] * r2[2]);
#pragma unroll
        for (int i = 0; i < 3; ++i) { r3[i] /= n3; r2[i] /= n2; }
        r1[0] = r2[1] * r3[2] - r2[2] * r3[1];
        r1[1] = r2[2] * r3[0] - r2[0] * r3[2];
        r1[2] = r2[0] * r3[1] - r2[1] * r3[0];
        const float sqrt2 = 1.4142135623730950488016887242097f;
        float2 R1[9];
        R1[0] = make_float2((r2[1] + r1[0]) * 0.5f, (r1[1] - r2[0]) * 0.5f);   // (-1,-1)
        R1[1] = make_float2(r3[0] / sqrt2, r3[1] / sqrt2);                    // (-1, 0)
        R1[2] = make_float2((r2[1] - r1[0]) * 0.5f, (-r1[1] - r2[0]) * 0.5f);  // (-1, 1)
        R1[3] = make_float2(r1[2] / sqrt2, -r2[2] / sqrt2);                   // ( 0,-1)
        R1[4] = make_float2(r3[2], 0.f);                                      // ( 0, 0)
        R1[5] = make_float2(-r1[2] / sqrt2, -r2[2] / sqrt2);                  // ( 0, 1)
        R1[6] = make_float2((r2[1] - r1[0]) * 0.5f, (r1[1] + r2[0]) * 0.5f);   // ( 1,-1)
        R1[7] = make_float2(-r3[0] / sqrt2, r3[1] / sqrt2);                   // ( 1, 0)
        R1[8] = make_float2((r2[1] + r1[0]) * 0.5f, (r2[0] - r1[1]) * 0.5f);   // ( 1, 1)
        // e^{-i alpha} = (qx - i qy) / |q_xy| (1 along z), and its powers
        const float rho = sqrtf((float)(qx * qx + qy * qy));
        const float2 e1 = rho > 0.f ? make_float2((float)qx / rho, -(float)qy / rho) : make_float2(1.f, 0.f);
        ph[0] = make_float2(1.f, 0.f);
#pragma unroll
        for (int k = 1; k <= MM; ++k) ph[k] = make_float2(ph[k - 1].x * e1.x - ph[k - 1].y * e1.y, ph[k - 1].x * e1.y + ph[k - 1].y * e1.x);
        // D^1(x, .) = Re(R^1(x, .) e^{+i x alpha}): x = -1 multiplies by e^{-i alpha}, x = 1 by its conjugate
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const float2 a0 = R1[j], a2 = R1[6 + j];
            D1[j] = a0.x * e1.x - a0.y * e1.y;      // x = -1
            D1[3 + j] = R1[3 + j].x;                // x = 0
            D1[6 + j] = a2.x * e1.x + a2.y * e1.y;  // x = 1: Re(a2 conj(e1))
        }
    }
    float Dh[NH];
    if constexpr (MM >= 2) {
#pragma unroll
        for (int l = 2; l <= MM; ++l) {
#pragma unroll
            for (int m = -l; m <= l; ++m) {
#pragma unroll
                for (int m1 = S::m1min(m); m1 <= l; ++m1) {
                    const int e = S::hidx(l, m, m1);
                    const int l1 = l - 1;
                    float val = 0.f;
                    auto term = [&](int tt, int xm, int xm1, int um, int um1) {
                        if (um < -l1 || um > l1 || um1 < -l1 || um1 > l1) return;
                        val += pp.rc[3 * e + tt] * D1[(xm + 1) * 3 + (xm1 + 1)] * ozd_dget<MM, MR, NH>(D1, Dh, l1, um, um1);
                    };
                    if (m1 < l) {
                        if (m == -l) term(0, -1, 0, m + 1, m1);
                        else if (m == l) term(0, 1, 0, m - 1, m1);
                        else { term(0, 0, 0, m, m1); term(1, 1, 0, m - 1, m1); term(2, -1, 0, m + 1, m1); }
                    } else {
                        if (m == -l) term(0, -1, 1, m + 1, m1 - 1);
                        else if (m == l) term(0, 1, 1, m - 1, m1 - 1);
                        else { term(0, 0, 1, m, m1 - 1); term(1, 1, 1, m - 1, m1 - 1); term(2, -1, 1, m + 1, m1 - 1); }
                    }
                    Dh[e] = val;
                }
            }
        }
    }
    auto phase = [&](int mu) {  // e^{-i mu alpha}
        const float2 p = ph[mu < 0 ? -mu : mu];
        return mu < 0 ? make_float2(p.x, -p.y) : p;
    };

    // ---- forward rotation (:505-523): t = drho e^{-i mu' alpha}, then the real D ----
#pragma unroll
    for (int m = 0; m <= MM; ++m)
#pragma unroll
        for (int mu2 = 0; mu2 <= m / MR; ++mu2) {
            float2 tq[2 * MM + 1], tm[2 * MM + 1];
#pragma unroll
            for (int mup = -m; mup <= m; ++mup) {
                const size_t off = (size_t)S::pidx(m, mup, mu2) * a.N;
                const float2 p = phase(mup), x = planes[off + kq], y = planes[off + km];
                tq[mup + m] = make_float2(x.x * p.x - x.y * p.y, x.x * p.y + x.y * p.x);
                tm[mup + m] = make_float2(y.x * p.x - y.y * p.y, y.x * p.y + y.y * p.x);
            }
            const float sg = (m & 1) ? -1.f : 1.f;
#pragma unroll
            for (int khi = -m; khi <= m; ++khi) {
                float2 s = make_float2(0.f, 0.f), u = make_float2(0.f, 0.f);
#pragma unroll
                for (int mup = -m; mup <= m; ++mup) {
                    const float d = ozd_dget<MM, MR, NH>(D1, Dh, m, mup, khi), dm = ozd_dget<MM, MR, NH>(D1, Dh, m, mup, -khi);
                    s.x = fmaf(tq[mup + m].x, d, s.x);
                    s.y = fmaf(tq[mup + m].y, d, s.y);
                    u.x = fmaf(tm[mup + m].x, dm, u.x);
                    u.y = fmaf(tm[mup + m].y, dm, u.y);
                }
                const int o = S::pidx(m, khi, mu2);
                sq[o * B] = s;
                smq[o * B] = make_float2(sg * u.x, sg * u.y);
            }
        }

    // ---- interpolated c (:534-539) and the OZ sums (:561-606), as k_ozp ----
    const double nrm = sqrt(qx * qx + qy * qy + qz * qz);
    const double eff = nrm / a.dq + 1.0;
    const int iq = (int)eff;
    const float alpha = (float)(eff - iq);
    const float2 *c0 = ctab + (size_t)(iq - 1) * a.ncoef;
    const float2 *c1 = ctab + (size_t)iq * a.ncoef;
    const float2 *crow = nullptr;
    if (cq) {
        const int sx = ix <= a.nx / 2 ? ix : ix - a.nx, sy = iy <= a.ny / 2 ? iy : iy - a.ny, sz = iz <= a.nz / 2 ? iz : iz - a.nz;
        crow = cq + (size_t)(sx * sx + sy * sy + sz * sz) * a.ncoef;
    }
#pragma unroll
    for (int khi = -MM; khi <= MM; ++khi) {
        constexpr int BMAX = 2 * (MM / MR + 1) * (MM + 1);
        float2 gs[BMAX], gm[BMAX];
        int nb = 0;
#pragma unroll
        for (int m = (khi < 0 ? -khi : khi); m <= MM; ++m)
#pragma unroll
            for (int mu2 = 0; mu2 <= m / MR; ++mu2) {
                const int ip = S::pidx(m, khi, mu2);
                float2 s = make_float2(0.f, 0.f), u = make_float2(0.f, 0.f);
                int k = 0;
#pragma unroll
                for (int n = (khi < 0 ? -khi : khi); n <= MM; ++n)
#pragma unroll
                    for (int nu2 = -n / MR; nu2 <= n / MR; ++nu2, ++k) {
                        const int ia = pp.ia0[ip] + k;
                        float2 ce;
                        if (crow) {
                            ce = crow[ia];
                        } else {
                            const float2 A0 = c0[ia], A1 = c1[ia];
                            ce.x = alpha * A1.x + (1.f - alpha) * A0.x;
                            ce.y = alpha * A1.y + (1.f - alpha) * A0.y;
                        }
                        const int jp = S::pidx(n, khi, nu2 < 0 ? -nu2 : nu2);
                        if (nu2 < 0) {
                            ozp_fma(s, ce, sq[jp * B]);
                            ozp_fma(u, ce, smq[jp * B]);
                        } else {
                            ozp_fmac(s, ce, smq[jp * B]);
                            ozp_fmac(u, ce, sq[jp * B]);
                        }
                    }
                gs[nb] = s;
                gm[nb] = u;
                ++nb;
            }
        nb = 0;
#pragma unroll
        for (int m = (khi < 0 ? -khi : khi); m <= MM; ++m)
#pragma unroll
            for (int mu2 = 0; mu2 <= m / MR; ++mu2) {
                const int ip = S::pidx(m, khi, mu2);
                sq[ip * B] = gs[nb];
                smq[ip * B] = gm[nb];
                ++nb;
            }
    }

    // ---- back rotation with conj(R) = e^{+i mu' alpha} D (:611-641), straight to the planes ----
#pragma unroll
    for (int m = 0; m <= MM; ++m)
#pragma unroll
        for (int mu2 = 0; mu2 <= m / MR; ++mu2) {
            float2 g[2 * MM + 1], gmv[2 * MM + 1];
#pragma unroll
            for (int k = -m; k <= m; ++k) {
                g[k + m] = sq[S::pidx(m, k, mu2) * B];
                gmv[k + m] = smq[S::pidx(m, k, mu2) * B];
            }
            const float sg = (m & 1) ? -1.f : 1.f;
#pragma unroll
            for (int khi = -m; khi <= m; ++khi) {  // output (m, mup = khi, mu2)
                float2 s = make_float2(0.f, 0.f), u = make_float2(0.f, 0.f);
#pragma unroll
                for (int k = -m; k <= m; ++k) {
                    const float d = ozd_dget<MM, MR, NH>(D1, Dh, m, khi, k), dm = ozd_dget<MM, MR, NH>(D1, Dh, m, khi, -k);
                    s.x = fmaf(g[k + m].x, d, s.x);
                    s.y = fmaf(g[k + m].y, d, s.y);
                    u.x = fmaf(gmv[k + m].x, dm, u.x);
                    u.y = fmaf(gmv[k + m].y, dm, u.y);
                }
                const float2 p = phase(-khi);  // e^{+i mup alpha}
                s = make_float2(s.x * p.x - s.y * p.y, s.x * p.y + s.y * p.x);
                u = make_float2(sg * (u.x * p.x - u.y * p.y), sg * (u.x * p.y + u.y * p.x));
                if (selfconj && nyq) u.y = -u.y;
                const size_t off = (size_t)S::pidx(m, khi, mu2) * a.N;
                if (!selfconj) planes[off + kq] = s;
                planes[off + km] = u;
            }
        }
}

inline size_t ozp_smem_bytes(int np) { return sizeof(float2) * 2 * (size_t)np * kOzpThreads; }

// c(|q|) interpolated on the host at every |q|^2 of a cubic grid in a cubic box (s2 = 0 ..
// 3 (n/2)^2, |q| = 2 pi/L sqrt(s2)), with the kernel's interpolation rule; empty otherwise.
inline std::vector<float2> build_ozp_cq(const Grid &g, const CTable &ct, const std::vector<float2> &c32) {
    std::vector<float2> t;
    if (!(g.nx == g.ny && g.ny == g.nz && g.lx == g.ly && g.ly == g.lz)) return t;
    const int h = g.nx / 2, rows = 3 * h * h + 1, nc = ct.ncoef;
    const double tp = 2.0 * kPi / g.lx;
    t.resize((size_t)rows * nc);
    for (int s2 = 0; s2 < rows; ++s2) {
        const double nrm = std::sqrt((double)s2) * tp;
        const double eff = nrm / ct.dq + 1.0;
        const int iq = (int)eff;
        if (iq < 1 || iq >= ct.nq) return std::vector<float2>();
        const float alpha = (float)(eff - iq);
        for (int i = 0; i < nc; ++i) {
            const float2 A = c32[(size_t)(iq - 1) * nc + i], B = c32[(size_t)iq * nc + i];
            t[(size_t)s2 * nc + i] = make_float2(alpha * B.x + (1.f - alpha) * A.x, alpha * B.y + (1.f - alpha) * A.y);
        }
    }
    return t;
}

// Host: parameters of k_ozp for this grid and c table; false when the shape is not covered
// (then k_oz2<float> runs).  The coefficients and term order mirror build_oz_tables.
inline bool build_ozp_params(const Grid &g, const CTable &ct, OzpParams &p) {
    if (g.np > kOzpMaxNp) return false;
    std::memset(&p, 0, sizeof p);
    for (int o = 0; o < g.np; ++o) p.ia0[o] = ct.ia_start[o];
    RotCoef rc;
    build_rot_coef(rc);
    int e = 0;
    for (int l = 2; l <= g.mmax; ++l)
        for (int m = -l; m <= l; ++m)
            for (int m1 = (m > 0 ? 1 : 0); m1 <= l; ++m1, ++e) {
                if (e >= kOzpMaxRec) return false;
                double c[3] = {0, 0, 0};
                if (m1 < l) {
                    if (m == -l) c[0] = rc.b[l][-m + kRMax][m1 + kRMax];
                    else if (m == l) c[0] = rc.b[l][m + kRMax][m1 + kRMax];
                    else {
                        c[0] = rc.a[l][m + kRMax][m1 + kRMax];
                        c[1] = rc.b[l][m + kRMax][m1 + kRMax];
                        c[2] = rc.b[l][-m + kRMax][m1 + kRMax];
                    }
                } else {
                    if (m == -l) c[0] = rc.d[l][-m + kRMax];
                    else if (m == l) c[0] = rc.d[l][m + kRMax];
                    else {
                        c[0] = rc.c[l][m + kRMax];
                        c[1] = rc.d[l][m + kRMax];
                        c[2] = rc.d[l][-m + kRMax];
                    }
                }
                for (int t = 0; t < 3; ++t) p.rc[3 * e + t] = (float)c[t];
            }
    return true;
}

}  // namespace mdft
