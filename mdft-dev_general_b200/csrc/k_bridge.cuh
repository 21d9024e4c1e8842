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

// n(r) into dens and into the real part of plane: one warp per grid point, the lanes
// striding over its orientations (coalesced), summed by shuffles
__global__ void __launch_bounds__(kBrThreads) k_cgb_density(const double *__restrict__ xi, const double *__restrict__ w, CgbArgs a,
                                                            double *__restrict__ dens, double2 *__restrict__ plane) {
    const int lane = threadIdx.x & 31;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long r = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < a.N; r += nw) {
        const double *x = xi + r * a.no;
        double s = 0.0;
        for (int io = lane; io < a.no; io += 32) s += x[io] * x[io] * a.rho0 * w[io];
        for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
        if (lane == 0) {
            const double n = s / a.n0;
            dens[r] = n;
            plane[r] = make_double2(n, 0.0);
        }
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

// ---------------------------------------------------------------------------------------
// Hard-sphere bridge, bridge = "hard_sphere" (src/module_fmt.f90:5-317, one species, FP64):
//   rho(r)   = sum_io xi^2 w                      wd_a = IFFT(FFT(rho) rho0 fl(w_a(|k|))) / N
//   F_b      = kT dv sum_r Phi(wd) - mu N_mol - Fexc0 - F_int      (PY or CS Phi)
//   df      += 2 xi rho0 (kT IFFT(sum_a FFT(dPhi/dwd_a) w_a) / N - mu) w
//   F_int, df -= the quadratic part of the hard-sphere c(k) (:223-282): gamma = IFFT(FFT(rho -
//   8 pi^2 / mrso) c_hs(k bin)) / N, F_int = sum w dv rho0 0.5 (xi^2 - 1) (-kT rho0 gamma),
//   df -= 2 xi w dv rho0 (-kT rho0 gamma) / dv.
// fl(): the reference's cmplx(w_k, 0) is single precision (:92).  Planes (N complex each):
// 0 rho, 1 rho - 8 pi^2/mrso (then gamma), 2-5 wd_a (then dPhi/dwd_a), 6 the gradient sum.
struct FmtArgs {
    long long N;
    int no, nx, ny, nz, version;  // 1 PY, 2 CS
    double rho0, kT, dv, R, mu, fexc0, shift, nd, dq;
    double lx, ly, lz;
    int nbk;
};

// |k| as norm_k (src/module_grid.f90:305-330): k = (l-1) 2 pi / L on the signed index
__device__ __forceinline__ double fmt_knorm(const FmtArgs &a, long long i) {
    const double twopi = 2.0 * kPi;
    const int ix = (int)(i % a.nx), iy = (int)((i / a.nx) % a.ny), iz = (int)(i / ((long long)a.nx * a.ny));
    const double kx = (double)(ix <= a.nx / 2 ? ix : ix - a.nx) * twopi / a.lx;
    const double ky = (double)(iy <= a.ny / 2 ? iy : iy - a.ny) * twopi / a.ly;
    const double kz = (double)(iz <= a.nz / 2 ? iz : iz - a.nz) * twopi / a.lz;
    return sqrt(kx * kx + ky * ky + kz * kz);
}

// w_a(k) of src/module_hardspheres.f90:56-70
__device__ __forceinline__ void fmt_weights(double R, double k, double w[4]) {
    const double fourpi = 4.0 * kPi;
    if (fabs(k) > kEpsDp) {
        const double kR = k * R, sk = sin(kR), ck = cos(kR);
        w[3] = fourpi * (sk - kR * ck) / (k * k * k);
        w[2] = fourpi * R * sk / k;
        w[1] = (sk + kR * ck) / (2 * k);
        w[0] = ck + kR * sk / 2;
    } else {
        w[3] = fourpi / 3 * (R * R * R);
        w[2] = fourpi * (R * R);
        w[1] = R;
        w[0] = 1;
    }
}

// planes 0, 1 <- rho, rho - shift; part[2 blk] = {sum rho, max |xi|}.  One warp per grid
// point, the lanes striding over its orientations (coalesced), summed by shuffles.
__global__ void __launch_bounds__(kBrThreads) k_fmt_density(const double *__restrict__ xi, const double *__restrict__ w, FmtArgs a,
                                                            double2 *__restrict__ pl, double *__restrict__ part) {
    __shared__ double sh[kBrThreads / 32];
    double srho = 0.0, mx = 0.0;
    const int lane = threadIdx.x & 31;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long r = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < a.N; r += nw) {
        const double *x = xi + r * a.no;
        double s = 0.0;
        for (int io = lane; io < a.no; io += 32) {
            s = s + x[io] * x[io] * w[io];
            mx = fmax(mx, fabs(x[io]));
        }
        for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
        if (lane == 0) {
            pl[r] = make_double2(s, 0.0);
            pl[a.N + r] = make_double2(s - a.shift, 0.0);
            srho += s;
        }
    }
    const double t = block_sum(srho, sh);
    __syncthreads();
    for (int off = 16; off > 0; off >>= 1) mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, off));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int i = 0; i < kBrThreads / 32; ++i) m = fmax(m, sh[i]);
        part[2 * blockIdx.x] = t;
        part[2 * blockIdx.x + 1] = m;
    }
}

// in k-space: planes 2-5 <- FFT(rho) rho0 fl(w_a); plane 1 <- FFT(rho - shift) c_hs(bin)
__global__ void k_fmt_weigh(double2 *__restrict__ pl, const double *__restrict__ cs, FmtArgs a) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.N; i += (long long)gridDim.x * blockDim.x) {
        const double k = fmt_knorm(a, i);
        double w[4];
        fmt_weights(a.R, k, w);
        const double2 r = pl[i];
        for (int c = 0; c < 4; ++c) {
            const double wf = (double)__double2float_rn(w[c]);
            pl[(2 + c) * a.N + i] = make_double2(r.x * a.rho0 * 1.0 * wf, r.y * a.rho0 * 1.0 * wf);
        }
        const int kb = min((int)(k / a.dq) + 1, a.nbk);
        const double c = cs[kb - 1];
        const double2 e = pl[a.N + i];
        pl[a.N + i] = make_double2(e.x * c, e.y * c);
    }
}

// wd_a = plane(2+a).x / N; Phi sums (PY: sum wd0 log(1-wd3), sum wd1 wd2/(1-wd3),
// sum wd2^3/(1-wd3)^2; CS: the three sums of :107-112); with want_g, planes 2-5 <- dPhi/dwd_a.
// part[4 blk] = {s1, s2, s3, error}: 1 wd3 >= 1, 2 (CS) wd3 <= eps, 3 (gradient) 1 - wd3 or wd3 at 0.
__global__ void __launch_bounds__(kBrThreads) k_fmt_phi(double2 *__restrict__ pl, FmtArgs a, int want_g, double *__restrict__ part) {
    __shared__ double sh[kBrThreads / 32];
    double s1 = 0.0, s2 = 0.0, s3 = 0.0, err = 0.0;
    const double i36 = 1.0 / (36.0 * kPi), i12 = 1.0 / (12.0 * kPi), i18 = 1.0 / (18.0 * kPi), i8 = 1.0 / (8.0 * kPi);
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < a.N; r += (long long)gridDim.x * blockDim.x) {
        const double w0 = pl[2 * a.N + r].x / a.nd, w1 = pl[3 * a.N + r].x / a.nd;
        const double w2 = pl[4 * a.N + r].x / a.nd, w3 = pl[5 * a.N + r].x / a.nd;
        if (w3 >= 1) err = fmax(err, 1.0);
        if (a.version == 2 && w3 <= kEpsDp) err = fmax(err, 2.0);
        const double u = 1 - w3, lg = log(u);
        if (a.version == 1) {
            s1 += w0 * lg;
            s2 += w1 * w2 / u;
            s3 += (w2 * w2 * w2) / (u * u);
        } else {
            s1 += w1 * w2 / u;
            s2 += (i36 * (w2 * w2 * w2) / (w3 * w3) - w0) * lg;
            s3 += i36 * (w2 * w2 * w2) / (w3 * (u * u));
        }
        if (want_g) {
            if (u <= kEpsDp || (a.version == 2 && fabs(w3) <= kEpsDp)) err = fmax(err, 3.0);
            double d0, d1, d2, d3;
            d0 = -lg;
            d1 = w2 / u;
            if (a.version == 1) {
                d2 = w1 / u + i8 * (d1 * d1);
                d3 = (w0 + w1 * d1) / u + i12 * (d1 * d1 * d1);
            } else {
                const double q = w2 / w3;
                d2 = -i12 * (q * q) * d0 + w1 / u + i12 * (d1 * d1) / w3;
                d3 = i18 * d0 * (q * q * q) - (i36 * (w2 * w2 * w2) / (w3 * w3) - w0) / u + w1 * d1 / u +
                     i36 * (w2 * w2 * w2) / (w3 * w3) * (3.0 * w3 - 1.0) / (u * u * u);
            }
            pl[2 * a.N + r] = make_double2(d0, 0.0);
            pl[3 * a.N + r] = make_double2(d1, 0.0);
            pl[4 * a.N + r] = make_double2(d2, 0.0);
            pl[5 * a.N + r] = make_double2(d3, 0.0);
        }
    }
    const double t1 = block_sum(s1, sh);
    __syncthreads();
    const double t2 = block_sum(s2, sh);
    __syncthreads();
    const double t3 = block_sum(s3, sh);
    __syncthreads();
    for (int off = 16; off > 0; off >>= 1) err = fmax(err, __shfl_down_sync(0xffffffffu, err, off));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = err;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int i = 0; i < kBrThreads / 32; ++i) m = fmax(m, sh[i]);
        part[4 * blockIdx.x + 0] = t1;
        part[4 * blockIdx.x + 1] = t2;
        part[4 * blockIdx.x + 2] = t3;
        part[4 * blockIdx.x + 3] = m;
    }
}

// plane 6 <- sum_a FFT(dPhi/dwd_a) w_a (FP64 weights, :170-174)
__global__ void k_fmt_combine(double2 *__restrict__ pl, FmtArgs a) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.N; i += (long long)gridDim.x * blockDim.x) {
        double w[4];
        fmt_weights(a.R, fmt_knorm(a, i), w);
        double2 s = make_double2(0.0, 0.0);
        for (int c = 0; c < 4; ++c) {
            const double2 v = pl[(2 + c) * a.N + i];
            s.x = (c == 0) ? v.x * w[c] : s.x + v.x * w[c];
            s.y = (c == 0) ? v.y * w[c] : s.y + v.y * w[c];
        }
        pl[6 * a.N + i] = s;
    }
}

// F_int partials, and with df (skipped for an empty box, stats[1] <= eps) the gradient update
// and the gather's reductions of the final gradient: part2[4 blk] = {df.dvec, max|df|, sum w df, F_int}.
__global__ void __launch_bounds__(kBrThreads) k_fmt_grad(const double *__restrict__ xi, const double *__restrict__ w, FmtArgs a,
                                                         const double2 *__restrict__ pl, const double *__restrict__ stats,
                                                         double *__restrict__ df, const double *__restrict__ dvec,
                                                         double *__restrict__ part2) {
    __shared__ double sh[kBrThreads / 32];
    double gdv = 0.0, gmx = 0.0, gun = 0.0, fint = 0.0;
    const bool upd = df && stats[1] > kEpsDp;
    const double fact = a.dv * a.rho0;
    const long long n = a.N * a.no;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const long long r = e / a.no;
        const int io = (int)(e - r * a.no);
        const double psi = xi[e], wio = w[io];
        const double vint = -a.kT * a.rho0 * (pl[a.N + r].x / a.nd);
        fint += wio * fact * 0.5 * (psi * psi - 1.0) * vint;
        if (df) {
            double g = df[e];
            if (upd) {
                const double dfex = pl[6 * a.N + r].x / a.nd;
                g = g + 2 * psi * a.rho0 * (a.kT * dfex - a.mu) * wio;
                g = g - 2.0 * psi * wio * fact * vint / a.dv;
                df[e] = g;
            }
            if (dvec) gdv = fma(g, dvec[e], gdv);
            gmx = fmax(gmx, fabs(g));
            gun = fma(g, wio, gun);
        }
    }
    const double t0 = block_sum(gdv, sh);
    __syncthreads();
    const double t2 = block_sum(gun, sh);
    __syncthreads();
    const double t3 = block_sum(fint, sh);
    __syncthreads();
    for (int off = 16; off > 0; off >>= 1) gmx = fmax(gmx, __shfl_down_sync(0xffffffffu, gmx, off));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = gmx;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int i = 0; i < kBrThreads / 32; ++i) m = fmax(m, sh[i]);
        part2[4 * blockIdx.x + 0] = t0;
        part2[4 * blockIdx.x + 1] = m;
        part2[4 * blockIdx.x + 2] = t2;
        part2[4 * blockIdx.x + 3] = t3;
    }
}

// stats = {sum rho, max |xi|} from k_fmt_density's partials (one block, fixed order)
__global__ void __launch_bounds__(kBrThreads) k_fmt_stats(const double *__restrict__ part, int nblk, double *__restrict__ stats) {
    __shared__ double sh[kBrThreads / 32];
    double s = 0.0, mx = 0.0;
    for (int i = threadIdx.x; i < nblk; i += blockDim.x) {
        s += part[2 * i];
        mx = fmax(mx, part[2 * i + 1]);
    }
    const double t = block_sum(s, sh);
    __syncthreads();
    for (int off = 16; off > 0; off >>= 1) mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, off));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int i = 0; i < kBrThreads / 32; ++i) m = fmax(m, sh[i]);
        stats[0] = t;
        stats[1] = m;
    }
}

// sums[6] = F_b, sums[7] = error code (0 for an empty box); with have_g, sums[3..5] too.
__global__ void __launch_bounds__(kBrThreads) k_fmt_finish(const double *__restrict__ part, const double *__restrict__ part2, int nblk,
                                                           const double *__restrict__ stats, FmtArgs a, int have_g,
                                                           double *__restrict__ sums) {
    __shared__ double sh[kBrThreads / 32];
    double v[7] = {0, 0, 0, 0, 0, 0, 0};  // s1 s2 s3 err | gdv gmx gun, then fint below
    double fint = 0.0;
    for (int i = threadIdx.x; i < nblk; i += blockDim.x) {
        v[0] += part[4 * i + 0];
        v[1] += part[4 * i + 1];
        v[2] += part[4 * i + 2];
        v[3] = fmax(v[3], part[4 * i + 3]);
        v[4] += part2[4 * i + 0];
        v[5] = fmax(v[5], part2[4 * i + 1]);
        v[6] += part2[4 * i + 2];
        fint += part2[4 * i + 3];
    }
    double t[8];
    const int sum_idx[5] = {0, 1, 2, 4, 6};
    for (int j = 0; j < 5; ++j) {
        t[sum_idx[j]] = block_sum(v[sum_idx[j]], sh);
        __syncthreads();
    }
    t[7] = block_sum(fint, sh);
    __syncthreads();
    for (int j : {3, 5}) {
        double m = v[j];
        for (int off = 16; off > 0; off >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, off));
        if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
        __syncthreads();
        if (threadIdx.x == 0) {
            double mm = 0.0;
            for (int i = 0; i < kBrThreads / 32; ++i) mm = fmax(mm, sh[i]);
            t[j] = mm;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const bool empty = !(stats[1] > kEpsDp);
        double f;
        if (empty) {
            f = -a.fexc0 * 1.0;
        } else {
            f = a.version == 1 ? -t[0] + t[1] + t[2] / (24 * kPi) : t[0] + t[1] + t[2];
            const double nmol = stats[0] * a.dv * a.rho0 * 1.0;
            f = f * a.kT * a.dv - a.mu * nmol - a.fexc0 * 1.0;
            f = f - t[7];
        }
        sums[6] = f;
        sums[7] = empty ? 0.0 : t[3];
        if (have_g) {
            sums[3] = t[4];
            sums[4] = t[5];
            sums[5] = t[6];
        }
    }
}

}  // namespace mdft
