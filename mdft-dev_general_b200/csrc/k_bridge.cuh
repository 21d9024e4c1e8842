// Coarse-grained bridge, bridge = "cgb" (src/module_coarse_grained_gageat_bridge.f90:50-482),
// for one species in FP64.  One evaluation:
//   n(r)    = sum_io xi^2 rho0 w(io) / n0            (integrate_over_orientations, :270-271)
//   n_cg    = c2r(r2c(n) K(k)) / N                   (:424-451)
//   'sla':  F_b = sum_r kT dv n0 Phi(n_cg),  g_cg = kT Phi'(n_cg)            (:274-347)
//   'wda':  F_b = sum_r kT dv n0 (n - 1) Phi(n_cg), g_cg = Phi'(n_cg)       (:349-419)
//   dfb     = c2r(r2c(g_cg) K(k)) / N
//   ('wda': dfb <- kT ((n - 1) dfb + Phi(n_cg)))
//   df     += 2 xi rho0 dfb w(io)                    (update_gradient, :455-482)
// K(k) is the forward transform of the normalised Gaussian of width sigma on the periodic grid
// (cut below 1e-10) times V / N (fill_kernel, :123-210).  The real transforms run as complex
// FFTs of real planes.  After the bridge has added to df, k_cgb_grad recomputes the gather's
// fused reductions (df.dvec, max|df|, sum w df) over the final gradient.
#pragma once

#include "common.cuh"

namespace mdft {

constexpr int kBrThreads = 256;

struct CgbArgs {
    long long N;
    int no, version;  // 1 'sla', 2 'wda'
    double rho0, n0, kT, vvox, nf;  // nf = real(N), single precision as the reference writes it
    double A3, B6;
};

// Phi(n_cg) and its derivative as the reference writes them for each version ('sla': the
// derivative times kT).
__device__ __forceinline__ void cgb_phi(const CgbArgs &a, double ncg, double &phib, double &d) {
    const double dn = ncg - 1.0, dn2 = dn * dn, dn3 = dn2 * dn;
    if (a.version == 1) {
        if (ncg < 1.0) {
            phib = a.A3 * dn3 + a.B6 * (ncg * ncg) * (dn2 * dn2);
            d = a.kT * a.A3 * 3.0 * dn2 + a.kT * a.B6 * (2.0 * ncg * (dn2 * dn2) + 4.0 * (ncg * ncg) * dn3);
        } else {
            phib = a.A3 * dn3;
            d = a.kT * a.A3 * 3.0 * dn2;
        }
    } else {
        if (ncg < 1.0) {
            phib = a.A3 * dn2 + a.B6 * (ncg * ncg) * dn3;
            d = a.A3 * 2.0 * dn + a.B6 * (2.0 * ncg * dn3 + 3.0 * (ncg * ncg) * dn2);
        } else {
            phib = a.A3 * dn2;
            d = a.A3 * 2.0 * dn;
        }
    }
}

// The Gaussian on the periodic grid (before its transform).
__global__ void k_cgb_kernel(double2 *__restrict__ kk, int nx, int ny, int nz, double dx, double dy, double dz, double gp,
                             double oo, double cut) {
    const long long n = (long long)nx * ny * nz;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int ix = (int)(i % nx), iy = (int)((i / nx) % ny), iz = (int)(i / ((long long)nx * ny));
        const double xp = dx * min(ix, nx - ix), yp = dy * min(iy, ny - iy), zp = dz * min(iz, nz - iz);
        const double d2 = xp * xp + yp * yp + zp * zp;
        kk[i] = make_double2(d2 < cut ? gp * exp(-d2 * oo) : 0.0, 0.0);
    }
}

// kk <- kk / nf * vol (fill_kernel's normalisation)
__global__ void k_cgb_scale(double2 *__restrict__ kk, long long n, double nf, double vol) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double2 v = kk[i];
        kk[i] = make_double2(v.x / nf * vol, v.y / nf * vol);
    }
}

// p <- p * kk (complex)
__global__ void k_cgb_cmul(double2 *__restrict__ p, const double2 *__restrict__ kk, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double2 a = p[i], b = kk[i];
        p[i] = make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
    }
}

// n(r) into dens and into the real part of plane (one thread per grid point)
__global__ void __launch_bounds__(kBrThreads) k_cgb_density(const double *__restrict__ xi, const double *__restrict__ w, CgbArgs a,
                                                            double *__restrict__ dens, double2 *__restrict__ plane) {
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < a.N; r += (long long)gridDim.x * blockDim.x) {
        const double *x = xi + r * a.no;
        double s = 0.0;
        for (int io = 0; io < a.no; ++io) s += x[io] * x[io] * a.rho0 * w[io];
        const double n = s / a.n0;
        dens[r] = n;
        plane[r] = make_double2(n, 0.0);
    }
}

__device__ __forceinline__ double block_sum(double s, double *sh) {
    for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int i = 0; i < kBrThreads / 32; ++i) t += sh[i];
    return t;
}

// F_b partial per block; with want_g, the derivative plane for the second convolution.
// ncg_plane holds N n_cg (the unnormalised inverse transform).
__global__ void __launch_bounds__(kBrThreads) k_cgb_phi(const double2 *__restrict__ ncg_plane, const double *__restrict__ dens,
                                                        CgbArgs a, int want_g, double2 *__restrict__ gplane,
                                                        double *__restrict__ part) {
    __shared__ double sh[kBrThreads / 32];
    double fb = 0.0;
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < a.N; r += (long long)gridDim.x * blockDim.x) {
        const double ncg = ncg_plane[r].x / a.nf;
        double phib, d;
        cgb_phi(a, ncg, phib, d);
        if (a.version == 1) fb += a.kT * a.vvox * a.n0 * phib;
        else fb += a.kT * a.vvox * a.n0 * (dens[r] - 1.0) * phib;
        if (want_g) gplane[r] = make_double2(d, 0.0);
    }
    const double t = block_sum(fb, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = t;
}

// df += 2 xi rho0 dfb w(io) over every (point, orientation), then the gather's reductions of
// the final gradient: part2[3 blk + {0,1,2}] = {df.dvec, max|df|, sum w df}.
__global__ void __launch_bounds__(kBrThreads) k_cgb_grad(const double *__restrict__ xi, const double *__restrict__ w, CgbArgs a,
                                                         const double2 *__restrict__ ncg_plane, const double2 *__restrict__ gplane,
                                                         const double *__restrict__ dens, double *__restrict__ df,
                                                         const double *__restrict__ dvec, double *__restrict__ part2) {
    __shared__ double sh[kBrThreads / 32];
    double gdv = 0.0, gmx = 0.0, gun = 0.0;
    const long long n = a.N * a.no;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const long long r = e / a.no;
        const int io = (int)(e - r * a.no);
        double dfb = gplane[r].x / a.nf;
        if (a.version == 2) {
            double phib, d;
            cgb_phi(a, ncg_plane[r].x / a.nf, phib, d);
            dfb = a.kT * ((dens[r] - 1.0) * dfb + phib);
        }
        const double g = df[e] + 2.0 * xi[e] * a.rho0 * dfb * w[io];
        df[e] = g;
        if (dvec) gdv = fma(g, dvec[e], gdv);
        gmx = fmax(gmx, fabs(g));
        gun = fma(g, w[io], gun);
    }
    const double s0 = block_sum(gdv, sh);
    __syncthreads();
    const double s2 = block_sum(gun, sh);
    __syncthreads();
    for (int off = 16; off > 0; off >>= 1) gmx = fmax(gmx, __shfl_down_sync(0xffffffffu, gmx, off));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = gmx;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int i = 0; i < kBrThreads / 32; ++i) m = fmax(m, sh[i]);
        part2[3 * blockIdx.x + 0] = s0;
        part2[3 * blockIdx.x + 1] = m;
        part2[3 * blockIdx.x + 2] = s2;
    }
}

// sums[6] = F_b; with nblk2 > 0 also sums[3..5] = the reductions of the final gradient.
// One block of kBrThreads, fixed order.
__global__ void __launch_bounds__(kBrThreads) k_cgb_finish(const double *__restrict__ part, int nblk, const double *__restrict__ part2,
                                                           int nblk2, double *__restrict__ sums) {
    __shared__ double sh[kBrThreads / 32];
    double fb = 0.0, gdv = 0.0, gun = 0.0, gmx = 0.0;
    for (int i = threadIdx.x; i < nblk; i += blockDim.x) fb += part[i];
    for (int i = threadIdx.x; i < nblk2; i += blockDim.x) {
        gdv += part2[3 * i + 0];
        gmx = fmax(gmx, part2[3 * i + 1]);
        gun += part2[3 * i + 2];
    }
    const double t0 = block_sum(fb, sh);
    __syncthreads();
    const double t1 = block_sum(gdv, sh);
    __syncthreads();
    const double t2 = block_sum(gun, sh);
    __syncthreads();
    for (int off = 16; off > 0; off >>= 1) gmx = fmax(gmx, __shfl_down_sync(0xffffffffu, gmx, off));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = gmx;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int i = 0; i < kBrThreads / 32; ++i) m = fmax(m, sh[i]);
        sums[6] = t0;
        if (nblk2 > 0) {
            sums[3] = t1;
            sums[4] = m;
            sums[5] = t2;
        }
    }
}

}  // namespace mdft
