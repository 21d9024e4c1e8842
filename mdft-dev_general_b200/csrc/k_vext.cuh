// External potential kernels (set-up, once per solute):
//  * Lennard-Jones on the grid nodes, src/module_lennardjones.f90:9-226, one
//    thread per node walking the solute sites in order (the reference skips a
//    node whose potential already exceeds 1e5, so the order matters);
//  * electrostatics, src/module_fastpoissonsolver.f90:121-288 with the solvent
//    charge factor of src/module_solvent.f90:367-438: V(k) = 4 pi rho(k)/k^2,
//    then for every orientation c2r( V(k) conj(sigma_k(io)) ) qfact / N;
//  * vext_total_sum, src/module_vext.f90:600-669.
#pragma once

#include "common.cuh"

namespace mdft {

struct LJTerm {
    double px, py, pz;   // solute site
    double epsuv, siguv6;
    double sx, sy, sz;   // solvent site in the molecular frame
    int lo[3][2], hi[3][2];  // node index intervals (0-based, inclusive; empty when lo > hi)
};

struct LJArgs {
    int nx, ny, nz, no;
    double dx, dy, dz, lx, ly, lz, cutoffsq;
    int nterm;
    int only_origin;
};

// How many times node index i occurs in the site's index table along one axis.
// The reference's wrapped table [1..max] ++ [min..n] holds one node twice when
// min == max (a cut-off cube as wide as the box); that node then gets the term twice.
__device__ __forceinline__ int multiplicity(const LJTerm &t, int ax, int i) {
    return (int)(i >= t.lo[ax][0] && i <= t.hi[ax][0]) + (int)(i >= t.lo[ax][1] && i <= t.hi[ax][1]);
}

__device__ __forceinline__ double pbc_dist(double d, double L) {
    d = fabs(d);
    while (d > L * 0.5) d = fabs(d - L);
    return d;
}

__device__ __forceinline__ double lj_value(double rsq, double cutoffsq, double epsuv, double siguv6) {
    if (rsq <= kEpsDp) return 1.79769313486231570815e308;  // huge(1._dp)
    if (rsq > cutoffsq) return 0.0;
    double div = siguv6 / (rsq * rsq * rsq);
    return 4.0 * epsuv * div * (div - 1.0);
}

// vext is [N][no]; terms in the reference's site order.
__global__ void k_lj(double *__restrict__ vext, const LJTerm *__restrict__ terms, const double *__restrict__ rotm, LJArgs a) {
    const long long N = (long long)a.nx * a.ny * a.nz;
    const long long total = a.only_origin ? N : N * a.no;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        const long long pt = a.only_origin ? e : e / a.no;
        const int io = a.only_origin ? 0 : (int)(e % a.no);
        const int ix = (int)(pt % a.nx), iy = (int)((pt / a.nx) % a.ny), iz = (int)(pt / ((long long)a.nx * a.ny));
        const double xg = ix * a.dx, yg = iy * a.dy, zg = iz * a.dz;
        double v = vext[pt * a.no + io];
        for (int u = 0; u < a.nterm; ++u) {
            const LJTerm t = terms[u];
            const int visits = multiplicity(t, 0, ix) * multiplicity(t, 1, iy) * multiplicity(t, 2, iz);
            if (visits == 0) continue;
            double xs = xg, ys = yg, zs = zg;
            if (!a.only_origin) {
                const double *R = rotm + 9 * io;
                xs += R[0] * t.sx + R[1] * t.sy + R[2] * t.sz;
                ys += R[3] * t.sx + R[4] * t.sy + R[5] * t.sz;
                zs += R[6] * t.sx + R[7] * t.sy + R[8] * t.sz;
            }
            double ddx = pbc_dist(xs - t.px, a.lx), ddy = pbc_dist(ys - t.py, a.ly), ddz = pbc_dist(zs - t.pz, a.lz);
            double rsq = ddx * ddx + ddy * ddy + ddz * ddz;
            const double vlj = lj_value(rsq, a.cutoffsq, t.epsuv, t.siguv6);
            for (int k = 0; k < visits; ++k)
                if (!(v > 1.e5)) v = v + vlj;  // nodes already above 1e5 are skipped
        }
        if (a.only_origin)
            for (int k = 0; k < a.no; ++k) vext[pt * a.no + k] = v;
        else
            vext[pt * a.no + io] = v;
    }
}

// real density -> complex plane
__global__ void k_real_to_cplx(const double *__restrict__ r, double2 *__restrict__ c, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        c[i] = make_double2(r[i], 0.0);
}

// V(k) = rho(k) 4 pi / k^2 with the index convention of poissonSolver (:206-238)
__global__ void k_poisson(const double2 *__restrict__ rk, double2 *__restrict__ vk, int nx, int ny, int nz, double lx,
                          double ly, double lz) {
    const long long N = (long long)nx * ny * nz;
    const double twopi = 2.0 * kPi, fourpi = 2.0 * twopi;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < N; e += (long long)gridDim.x * blockDim.x) {
        int i = (int)(e % nx), j = (int)((e / nx) % ny), k = (int)(e / ((long long)nx * ny));
        int m1 = (i + 1 <= nx / 2) ? i : i - nx;
        int m2 = (j + 1 <= ny / 2) ? j : j - ny;
        int m3 = (k + 1 <= nz / 2) ? k : k - nz;
        double a = twopi * m1 / lx, b = twopi * m2 / ly, c = twopi * m3 / lz;
        double k2 = a * a + b * b + c * c;
        double2 v = make_double2(0.0, 0.0);
        if (fabs(k2) > kEpsDp) {
            double2 r = rk[e];
            v = make_double2(r.x * fourpi / k2, r.y * fourpi / k2);
        }
        vk[e] = v;
    }
}

struct SigmaArgs {
    int nx, ny, nz, no;
    double twopi_lx, twopi_ly, twopi_lz;
    int nsite;       // charged solvent sites
    int io0, nbatch; // orientations of this batch
};

// planes[b][k] = full-spectrum X_io(k), io = io0 + b: V(k) conj(sigma_k(io)) on the
// kx <= nx/2 half and its Hermitian mirror elsewhere.
__global__ void k_sigma_product(const double2 *__restrict__ vk, double2 *__restrict__ planes, const double *__restrict__ rotm,
                                const double *__restrict__ sq, const double *__restrict__ sxyz, SigmaArgs a) {
    const long long N = (long long)a.nx * a.ny * a.nz;
    const long long total = N * a.nbatch;
    const double smoother = 0.5;  // src/module_solvent.f90:382
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(e / N);
        const long long kidx = e % N;
        const int io = a.io0 + b;
        int i = (int)(kidx % a.nx), j = (int)((kidx / a.nx) % a.ny), k = (int)(kidx / ((long long)a.nx * a.ny));
        bool mirror = i > a.nx / 2;
        if (mirror) {
            i = a.nx - i;
            j = (a.ny - j) % a.ny;
            k = (a.nz - k) % a.nz;
        }
        const double kx = (i <= a.nx / 2 ? i : i - a.nx) * a.twopi_lx;
        const double ky = (j <= a.ny / 2 ? j : j - a.ny) * a.twopi_ly;
        const double kz = (k <= a.nz / 2 ? k : k - a.nz) * a.twopi_lz;
        const double sm = exp(-smoother * smoother * (kx * kx + ky * ky + kz * kz) / 2.0);
        const double *R = rotm + 9 * io;
        double sre = 0.0, sim = 0.0;
        for (int s = 0; s < a.nsite; ++s) {
            const double *r = sxyz + 3 * s;
            double r0 = R[0] * r[0] + R[1] * r[1] + R[2] * r[2];
            double r1 = R[3] * r[0] + R[4] * r[1] + R[5] * r[2];
            double r2 = R[6] * r[0] + R[7] * r[1] + R[8] * r[2];
            double kr = kx * r0 + ky * r1 + kz * r2;
            double sn, cs;
            sincos(-kr, &sn, &cs);
            sre += sq[s] * cs * sm;
            sim += sq[s] * sn * sm;
        }
        const long long src = ((long long)k * a.ny + j) * a.nx + i;
        const double2 v = vk[src];
        // v * conj(sigma)
        double2 x = make_double2(v.x * sre + v.y * sim, v.y * sre - v.x * sim);
        if (mirror) x.y = -x.y;
        planes[(size_t)b * N + kidx] = x;
    }
}

// vextq[r][io0+b] = qfact Re(planes[b][r]) / N
__global__ void k_sigma_store(const double2 *__restrict__ planes, double *__restrict__ vq, int no, int io0, int nbatch,
                              long long N, double scale) {
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < N * nbatch; e += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(e % nbatch);
        const long long r = e / nbatch;
        vq[r * no + io0 + b] = scale * planes[(size_t)b * N + r].x;
    }
}

// vext = min(vext + vq, thr); flag[0] |= 1 on NaN/Inf, |= 2 when vext <= -thr
__global__ void k_vext_total(double *__restrict__ vext, const double *__restrict__ vq, double thr, long long n,
                             int *__restrict__ flag) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        double v = vext[i];
        if (vq) v = v + vq[i];
        if (v > thr) v = thr;
        if (v != v || isinf(v)) atomicOr(flag, 1);
        if (v <= -thr) atomicOr(flag, 2);
        vext[i] = v;
    }
}

// partial[blk] = sum_r sum_io xi^2 rho0 w(io)   (density integral of pressure_correction)
__global__ void __launch_bounds__(256) k_density_sum(const double *__restrict__ xi, const double *__restrict__ w, int no,
                                                     long long n, double rho0, double *__restrict__ part) {
    double s = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        double x = xi[i];
        s += x * x * rho0 * w[i % no];
    }
    __shared__ double ss[8];
    for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
    if ((threadIdx.x & 31) == 0) ss[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int i = 0; i < 8; ++i) t += ss[i];
        part[2 * blockIdx.x] = t;
        part[2 * blockIdx.x + 1] = 0.0;
    }
}

}  // namespace mdft
