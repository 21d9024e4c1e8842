// Learned warm start of a solve: the network's input channels from the solute, the
// training target from a converged density, and the starting density built from a
// prediction.  Included by solve.cuh (it uses the handle, lbfgs_alloc and kQfact).
//
// Channels (FP32, [3][N], point order of xi without io), on the solver's grid with
// points at (ix dx, iy dy, iz dz) and minimum-image distances d to each solute site:
//   0: Lennard-Jones energy of the solvent's LJ site, sum over sites with d <= rvdw of
//      4 e (s^2 - s), s = (sigma/d)^6, Lorentz-Berthelot mixing; asinh(min(v/kT, 1e4))/4;
//   1: electrostatic potential of the sites' charges, each a Gaussian of width 0.5 A
//      (qfact q erf(d / (sqrt2 0.5)) / d), in kT per unit charge; asinh(V/kT)/4;
//   2: site density, sum over sites of exp(-d^2 / (2 0.5^2)).
// Target (FP32, [4][N]): the m <= 1, psi-independent projections of the log-density
// f(omega) = ln(rho/rho0) = 2 ln xi, clamped to [-8, 4], in the real basis
// {1, u_x, u_y, u_z} with u = R(omega) z the molecular z axis in the lab frame:
//   a_0 = sum_io w f / sum_io w,   a_k = sum_io w f u_k / sum_io w u_k^2   (k = x, y, z),
// exact projections for the Gauss-Legendre x uniform-phi quadrature of mmax >= 1.  The
// complex projections p(m <= 1, mu', mu = 0) of the reference's angl2proj
// (src/module_orientation_projection_transform.f90:159-199) span the same functions.
// Projection form (networks with nout = 2 np): target [2 np][N] = the real and imaginary
// parts of the np complex projections of the same clamped f with the handle's angl2proj
// matrix A (src/module_orientation_projection_transform.f90:159-199), in the reference's
// projection order; the start expands a prediction with the handle's proj2angl matrix B
// (:202-243): f(omega) = sum_k pred_k B_k(omega), clamped and exponentiated as below.
// Mask (FP32, [N]): 1 where some orientation is outside the hard core (vext < vmax).
// Start: f = a_0 + a . u clamped to [-2, 4], xi = exp(f/2), and xi = 0 wherever
// guess_density puts 0 (vext >= vmax, src/module_density.f90:267-284).  The start's floor
// is above the target's: dF/dxi is proportional to xi, so a region started near xi = 0
// passes a max|df| test at the wrong density (a start floor of -8, xi = 0.018, left 28 of
// 200 held-out solves at a different stationary point, up to 25 kJ/mol away).
#pragma once

namespace {

struct WarmSite {
    double x, y, z, q, sig, eps;
};

struct WarmFeatArgs {
    int nx, ny, nz, nsite;
    double dx, dy, dz, lx, ly, lz;
    double sig_s, eps_s;  // the solvent's Lennard-Jones site
    double rvdw2, kT, qfact;
};

constexpr double kWarmSmear = 0.5;  // A, width of the charge and site Gaussians
constexpr double kWarmFloor = -8.0, kWarmCeil = 4.0;  // target clamp of ln(rho/rho0)
constexpr double kWarmStartFloor = -2.0;               // start clamp (xi >= exp(-1))

__global__ void k_warm_features(float *__restrict__ feat, const WarmSite *__restrict__ s, WarmFeatArgs a) {
    const long long N = (long long)a.nx * a.ny * a.nz;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N; p += (long long)gridDim.x * blockDim.x) {
        const int ix = (int)(p % a.nx);
        const long long t = p / a.nx;
        const int iy = (int)(t % a.ny), iz = (int)(t / a.ny);
        const double rx = ix * a.dx, ry = iy * a.dy, rz = iz * a.dz;
        double vlj = 0.0, vq = 0.0, dens = 0.0;
        for (int k = 0; k < a.nsite; ++k) {
            double dx = rx - s[k].x, dy = ry - s[k].y, dz = rz - s[k].z;
            dx -= a.lx * rint(dx / a.lx);
            dy -= a.ly * rint(dy / a.ly);
            dz -= a.lz * rint(dz / a.lz);
            const double r2 = dx * dx + dy * dy + dz * dz;
            if (s[k].eps > 0.0 && a.eps_s > 0.0 && r2 <= a.rvdw2) {
                if (r2 < 1e-6) {
                    vlj += 1e10;
                } else {
                    const double sg = 0.5 * (s[k].sig + a.sig_s), e = sqrt(s[k].eps * a.eps_s);
                    const double s2 = sg * sg / r2, s6 = s2 * s2 * s2;
                    vlj += 4.0 * e * (s6 * s6 - s6);
                }
            }
            if (s[k].q != 0.0) {
                const double r = sqrt(r2);
                vq += r < 1e-6 ? s[k].q * 0.79788456080286536 / kWarmSmear : s[k].q * erf(r * (0.70710678118654752 / kWarmSmear)) / r;
            }
            dens += exp(-r2 * (0.5 / (kWarmSmear * kWarmSmear)));
        }
        vq *= a.qfact;
        feat[p] = (float)(0.25 * asinh(fmin(vlj / a.kT, 1e4)));
        feat[N + p] = (float)(0.25 * asinh(vq / a.kT));
        feat[2 * N + p] = (float)dens;
    }
}

// dir[io] = {u_x, u_y, u_z, w}
__global__ void k_warm_target(const double *__restrict__ xi, const double *__restrict__ vext, const double4 *__restrict__ dir,
                              float *__restrict__ target, float *__restrict__ mask, int no, long long N, double vmax, double4 norm) {
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N; p += (long long)gridDim.x * blockDim.x) {
        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
        bool open = false;
        const double *x = xi + p * no;
        const double *v = vext + p * no;
        for (int io = 0; io < no; ++io) {
            const double xv = x[io];
            double f = xv > 0.0 ? 2.0 * log(xv) : kWarmFloor;
            f = fmin(fmax(f, kWarmFloor), kWarmCeil);
            const double4 d = dir[io];
            s0 += d.w * f;
            s1 += d.w * f * d.x;
            s2 += d.w * f * d.y;
            s3 += d.w * f * d.z;
            open = open || v[io] < vmax;
        }
        target[p] = (float)(s0 * norm.x);
        target[N + p] = (float)(s1 * norm.y);
        target[2 * N + p] = (float)(s2 * norm.z);
        target[3 * N + p] = (float)(s3 * norm.w);
        if (mask) mask[p] = open ? 1.f : 0.f;
    }
}

__global__ void k_warm_expand(const float *__restrict__ pred, const double *__restrict__ vext, const double4 *__restrict__ dir,
                              double *__restrict__ xi, int no, long long N, double vmax) {
    const long long n = N * no;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long p = i / no;
        const int io = (int)(i - p * no);
        const double4 d = dir[io];
        double f = (double)pred[p] + (double)pred[N + p] * d.x + (double)pred[2 * N + p] * d.y + (double)pred[3 * N + p] * d.z;
        f = fmin(fmax(f, kWarmStartFloor), kWarmCeil);
        xi[i] = vext[i] >= vmax ? 0.0 : exp(0.5 * f);
    }
}

// projection form: A is [no][2np] (angl2proj), one thread per point
__global__ void k_warm_target_proj(const double *__restrict__ xi, const double *__restrict__ vext, const double *__restrict__ A,
                                   float *__restrict__ target, float *__restrict__ mask, int no, int nk, long long N, double vmax) {
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N; p += (long long)gridDim.x * blockDim.x) {
        const double *x = xi + p * no;
        const double *v = vext + p * no;
        bool open = false;
        for (int io = 0; io < no; ++io) open = open || v[io] < vmax;
        for (int k = 0; k < nk; ++k) {
            double acc = 0.0;
            for (int io = 0; io < no; ++io) {
                const double xv = x[io];
                const double f = fmin(fmax(xv > 0.0 ? 2.0 * log(xv) : kWarmFloor, kWarmFloor), kWarmCeil);
                acc = fma(f, A[(size_t)io * nk + k], acc);
            }
            target[(size_t)k * N + p] = (float)acc;
        }
        if (mask) mask[p] = open ? 1.f : 0.f;
    }
}

// projection form: B is [2np][no] (proj2angl)
__global__ void k_warm_expand_proj(const float *__restrict__ pred, const double *__restrict__ vext, const double *__restrict__ B,
                                   double *__restrict__ xi, int no, int nk, long long N, double vmax) {
    const long long n = N * no;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long p = i / no;
        const int io = (int)(i - p * no);
        double f = 0.0;
        for (int k = 0; k < nk; ++k) f = fma((double)pred[(size_t)k * N + p], B[(size_t)k * no + io], f);
        f = fmin(fmax(f, kWarmStartFloor), kWarmCeil);
        xi[i] = vext[i] >= vmax ? 0.0 : exp(0.5 * f);
    }
}

double guess_vmax(const mdft_handle *h) { return (-std::log(kEpsDp) - (double)0.05f) * h->g.kT; }

// the output forms a handle accepts: 4 (m <= 1 real basis) or 2 np (all projections)
int check_warm_nout(const mdft_handle *h, int nout) {
    if (nout == 4 || nout == 2 * h->g.np) return MDFT_OK;
    set_error("warm-start output count %d: 4 (m <= 1) or %d (all projections of this grid)", nout, 2 * h->g.np);
    return MDFT_E_ARG;
}

int warm_tables(mdft_handle *h, double4 *norm);

// prediction -> starting density in d_xi, in the form of nout outputs
int warm_expand_any(mdft_handle *h, const float *pred, int nout, double *d_xi) {
    const Grid &g = h->g;
    if (nout == 4) {
        double4 norm;
        int rc = warm_tables(h, &norm);
        if (rc) return rc;
        k_warm_expand<<<vec_grid(), 256, 0, h->stream>>>(pred, h->vext.p, h->wdir.p, d_xi, g.no, g.N, guess_vmax(h));
    } else {
        k_warm_expand_proj<<<vec_grid(), 256, 0, h->stream>>>(pred, h->vext.p, h->B.p, d_xi, g.no, 2 * g.np, g.N, guess_vmax(h));
    }
    h->launches += 1;
    return check_cuda(cudaGetLastError(), "warm-start expand");
}

// {u_x, u_y, u_z, w} per orientation on the device, and the projection normalisations
int warm_tables(mdft_handle *h, double4 *norm) {
    const Grid &g = h->g;
    std::vector<double4> dir(g.no);
    double sw = 0.0, sx = 0.0, sy = 0.0, sz = 0.0;
    for (int io = 0; io < g.no; ++io) {
        const double *R = &g.rotm[9 * (size_t)io];
        dir[io] = make_double4(R[2], R[5], R[8], g.w[io]);
        sw += g.w[io];
        sx += g.w[io] * R[2] * R[2];
        sy += g.w[io] * R[5] * R[5];
        sz += g.w[io] * R[8] * R[8];
    }
    if (!(sx > 0.0 && sy > 0.0 && sz > 0.0)) {
        set_error("warm start needs mmax >= 1 (an orientation-dependent density)");
        return MDFT_E_ARG;
    }
    *norm = make_double4(1.0 / sw, 1.0 / sx, 1.0 / sy, 1.0 / sz);
    if (!h->wdir.p) {
        int rc = alloc_check(h->wdir.alloc(g.no), "warm-start orientations", g.no * sizeof(double4));
        if (rc) return rc;
        cudaMemcpyAsync(h->wdir.p, dir.data(), g.no * sizeof(double4), cudaMemcpyHostToDevice, h->stream);
    }
    return MDFT_OK;
}

int warm_features_impl(mdft_handle *h, int nsite, const double *q, const double *sig, const double *eps, const double *xyz, int nsv,
                       const double *ssig, const double *seps, double rvdw, float *d_feat) {
    const Grid &g = h->g;
    int rc;
    std::vector<WarmSite> s(std::max(nsite, 1));
    for (int k = 0; k < nsite; ++k) s[k] = WarmSite{xyz[3 * k], xyz[3 * k + 1], xyz[3 * k + 2], q[k], sig[k], eps[k]};
    double sig_s = 0.0, eps_s = 0.0;
    for (int k = 0; k < nsv; ++k)
        if (seps[k] > 0.0) { sig_s = ssig[k]; eps_s = seps[k]; break; }
    if (h->wsite.n < s.size() * 6) {
        if ((rc = alloc_check(h->wsite.alloc(std::max<size_t>(s.size(), 64) * 6), "warm-start sites", s.size() * 48))) return rc;
    }
    cudaMemcpyAsync(h->wsite.p, s.data(), s.size() * sizeof(WarmSite), cudaMemcpyHostToDevice, h->stream);
    WarmFeatArgs a{g.nx, g.ny, g.nz, nsite, g.dx, g.dy, g.dz, g.lx, g.ly, g.lz, sig_s, eps_s, rvdw * rvdw, g.kT, kQfact};
    k_warm_features<<<vec_grid(), 256, 0, h->stream>>>(d_feat, reinterpret_cast<const WarmSite *>(h->wsite.p), a);
    h->launches += 1;
    // the host copy of the sites must outlive the asynchronous upload
    return check_cuda(cudaStreamSynchronize(h->stream), "warm-start features");
}

// the network's prediction for the handle's current solute -> starting density in d_xi
int warm_start_impl(mdft_handle *h, int nsite, const double *q, const double *sig, const double *eps, const double *xyz, int nsv,
                    const double *ssig, const double *seps, double rvdw, double *d_xi) {
    const Grid &g = h->g;
    int rc;
    double4 norm;
    if ((rc = warm_tables(h, &norm))) return rc;
    if (!h->wfeat.p && (rc = alloc_check(h->wfeat.alloc(3 * (size_t)g.N), "warm-start channels", 12 * (size_t)g.N))) return rc;
    if ((rc = warm_features_impl(h, nsite, q, sig, eps, xyz, nsv, ssig, seps, rvdw, h->wfeat.p))) return rc;
    long long before = 0, after = 0;
    mdft_warm_net_launch_count(h->warm, &before);
    if ((rc = mdft_warm_net_forward(h->warm, h->wfeat.p, nullptr))) return rc;
    mdft_warm_net_launch_count(h->warm, &after);
    h->launches += after - before;
    const float *pred = nullptr;
    if ((rc = mdft_warm_net_output(h->warm, &pred))) return rc;
    int nout = 4;
    if ((rc = mdft_warm_net_num_outputs(h->warm, &nout))) return rc;
    return warm_expand_any(h, pred, nout, d_xi);
}

}  // namespace

extern "C" {

int mdft_warm_features(mdft_handle *h, int nsite, const double *q, const double *sig, const double *eps, const double *xyz, int nsv,
                       const double *sq, const double *ssig, const double *seps, const double *sxyz, double rvdw, float *d_feat) {
    (void)sq;
    (void)sxyz;
    if (!h || !d_feat || nsite < 0 || (nsite > 0 && (!q || !sig || !eps || !xyz)) || nsv <= 0 || !ssig || !seps) {
        set_error("null or invalid argument");
        return MDFT_E_ARG;
    }
    return warm_features_impl(h, nsite, q, sig, eps, xyz, nsv, ssig, seps, rvdw, d_feat);
}

int mdft_warm_target(mdft_handle *h, const double *d_xi, float *d_target, float *d_mask) {
    return mdft_warm_target_n(h, d_xi, 4, d_target, d_mask);
}

int mdft_warm_target_n(mdft_handle *h, const double *d_xi, int nout, float *d_target, float *d_mask) {
    if (!h || !d_target) { set_error("null argument"); return MDFT_E_ARG; }
    int rc0 = check_warm_nout(h, nout);
    if (rc0) return rc0;
    if (!h->have_vext) { set_error("no vext yet"); return MDFT_E_STATE; }
    if (!d_xi) {
        if (!h->lb.x.p) { set_error("no solve has run on this handle"); return MDFT_E_STATE; }
        d_xi = h->lb.x.p;
    }
    const Grid &g = h->g;
    if (nout == 4) {
        double4 norm;
        int rc = warm_tables(h, &norm);
        if (rc) return rc;
        k_warm_target<<<vec_grid(), 256, 0, h->stream>>>(d_xi, h->vext.p, h->wdir.p, d_target, d_mask, g.no, g.N, guess_vmax(h), norm);
    } else {
        k_warm_target_proj<<<vec_grid(), 256, 0, h->stream>>>(d_xi, h->vext.p, h->A.p, d_target, d_mask, g.no, 2 * g.np, g.N,
                                                              guess_vmax(h));
    }
    h->launches += 1;
    return check_cuda(cudaGetLastError(), "warm-start target");
}

int mdft_warm_expand(mdft_handle *h, const float *d_pred, double *d_xi) { return mdft_warm_expand_n(h, d_pred, 4, d_xi); }

int mdft_warm_expand_n(mdft_handle *h, const float *d_pred, int nout, double *d_xi) {
    if (!h || !d_pred) { set_error("null argument"); return MDFT_E_ARG; }
    int rc0 = check_warm_nout(h, nout);
    if (rc0) return rc0;
    if (!h->have_vext) { set_error("no vext yet"); return MDFT_E_STATE; }
    if (!d_xi) {
        if (!h->lb.x.p) { set_error("no solve has run on this handle"); return MDFT_E_STATE; }
        d_xi = h->lb.x.p;
    }
    return warm_expand_any(h, d_pred, nout, d_xi);
}

int mdft_set_warm_net(mdft_handle *h, mdft_warm_net *net) {
    if (!h) { set_error("null handle"); return MDFT_E_ARG; }
    if (net) {
        int nxyz[3];
        int rc = mdft_warm_net_grid(net, nxyz);
        if (rc) return rc;
        if (nxyz[0] != h->g.nx || nxyz[1] != h->g.ny || nxyz[2] != h->g.nz) {
            set_error("warm-start network built for %dx%dx%d, handle grid %dx%dx%d", nxyz[0], nxyz[1], nxyz[2], h->g.nx, h->g.ny,
                      h->g.nz);
            return MDFT_E_ARG;
        }
        if (h->g.no < 2) { set_error("warm start needs mmax >= 1"); return MDFT_E_ARG; }
        int nout = 0;
        if ((rc = mdft_warm_net_num_outputs(net, &nout))) return rc;
        if ((rc = check_warm_nout(h, nout))) return rc;
    }
    cudaStreamSynchronize(h->stream);
    // a network that is detached goes back to its own stream
    if (h->warm && h->warm != net) mdft_warm_net_set_stream(h->warm, nullptr);
    if (net) {
        int rc = mdft_warm_net_set_stream(net, h->stream);
        if (rc) return rc;
    }
    h->warm = net;
    return MDFT_OK;
}

int mdft_get_warm_stats(const mdft_handle *h, long long *stats) {
    if (!h || !stats) { set_error("null argument"); return MDFT_E_ARG; }
    stats[0] = h->warm_starts;
    stats[1] = h->warm_fallbacks;
    return MDFT_OK;
}

}  // extern "C"
