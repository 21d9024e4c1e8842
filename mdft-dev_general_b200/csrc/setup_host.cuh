// Host-side set-up of an MDFT system: spatial grid and angular quadrature,
// projection index maps, Wigner small-d tables, dense angular transform
// matrices, and the c(k) table read from a Luc-format file.
#pragma once

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "common.cuh"

namespace mdft {

// sqrt(2m+1) except the reference's fm(7)=sqrt(14)
// (src/module_orientation_projection_transform.f90:35); m <= 5 here.
inline double fm_of(int m) { return std::sqrt(2.0 * m + 1.0); }

inline double factorial(int n) {
    double r = 1.0;
    for (int i = 2; i <= n; ++i) r *= (double)i;
    return r;
}

inline double powi(double x, int n) {
    double r = 1.0;
    for (int i = 0; i < n; ++i) r *= x;
    return r;
}

// Wigner small d^m_{mu,mup}(theta): src/module_wigner_d.f90:6-60.  For
// mu or mup = 0 the associated-Legendre recurrence, otherwise Wigner's sum.
inline double wigner_small_d(int m, int mu, int mup, double theta) {
    if (std::abs(mu) > m || std::abs(mup) > m) return 0.0;
    if (m == 0) return 1.0;
    if (mu == 0 || mup == 0) {
        int mu0 = (mu == 0) ? mup : mu;
        double th = (mu == 0) ? -theta : theta;
        double x = 1.0;
        if (mu0 < 0) {
            x = neg1pow(mu0);
            mu0 = -mu0;
        }
        double cc = std::cos(th), p_prev = 0.0, p = 1.0;
        for (int l = mu0 + 1; l <= m; ++l) {
            double pl = (cc * (2 * l - 1) * p - (double)(l + mu0 - 1) * p_prev) / (double)(l - mu0);
            p_prev = p;
            p = pl;
        }
        return x * neg1pow(mu0) * std::sqrt(factorial(m - mu0) / factorial(m + mu0)) * factorial(2 * mu0) /
               (powi(2.0, mu0) * factorial(mu0)) * powi(std::sin(th), mu0) * p;
    }
    double c = std::cos(0.5 * theta), s = std::sin(0.5 * theta), acc = 0.0;
    int lo = std::max(0, mu - mup), hi = std::min(m + mu, m - mup);
    for (int k = lo; k <= hi; ++k)
        acc += neg1pow(k) / (factorial(m + mu - k) * factorial(m - mup - k) * factorial(k) * factorial(k - mu + mup)) *
               powi(c, 2 * m + mu - mup - 2 * k) * powi(s, 2 * k - mu + mup);
    return std::sqrt(factorial(m + mu) * factorial(m - mu) * factorial(m + mup) * factorial(m - mup)) * acc;
}

// Gauss-Legendre nodes in cos(theta) and weights summing to one, by the Newton
// iteration of src/module_grid.f90:262-301.
inline void gauss_legendre(int n, std::vector<double> &x, std::vector<double> &w) {
    x.assign(n, 0.0);
    w.assign(n, 0.0);
    for (int i = 1; i <= (n + 1) / 2; ++i) {
        double z = std::cos(kPi * (i - 0.25) / (n + 0.5)), dz = 1.0, pd = 0.0;
        while (std::fabs(dz) > kEpsDp) {
            double p1 = 1.0, p2 = 0.0;
            for (int j = 1; j <= n; ++j) {
                double p3 = p2;
                p2 = p1;
                p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
            }
            pd = n * (z * p1 - p2) / (z * z - 1.0);
            dz = -p1 / pd;
            z += dz;
        }
        x[i - 1] = z;
        w[i - 1] = 1.0 / ((1.0 - z * z) * pd * pd);
        x[n - i] = -z;
        w[n - i] = w[i - 1];
    }
}

struct Grid {
    int nx = 0, ny = 0, nz = 0;
    long long N = 0;
    double lx = 0, ly = 0, lz = 0, dx = 0, dy = 0, dz = 0, dv = 0;
    int mmax = 0, mrso = 1, ntheta = 0, nphi = 0, npsi = 0, no = 0, np = 0, nmu2 = 0;
    double kT = 0, n0 = 0, rho0 = 0;
    std::vector<double> theta, wtheta, phi, psi, w;  // w[no]
    std::vector<double> rotm;                         // [no][9], row-major orientation matrices
    std::vector<int> pm, pmup, pmu;                   // projection -> (m, mup, mu)
    std::vector<double> wig;                          // [np][ntheta]
    std::vector<double> kx, ky, kz;                   // k components in FFTW order, Nyquist positive

    // ip of (m, mup, mu2) in the reference ordering: m, then mup = -m..m, then mu2 = 0..m/mrso.
    int pidx(int m, int mup, int mu2) const {
        int off = 0;
        for (int k = 0; k < m; ++k) off += (2 * k + 1) * (k / mrso + 1);
        return off + (mup + m) * (m / mrso + 1) + mu2;
    }
};

// src/module_grid.f90:51-212 with the projection tables of
// src/module_orientation_projection_transform.f90:80-133.
inline int build_grid(Grid &g, int nx, int ny, int nz, double lx, double ly, double lz, int mmax, int mrso,
                      double kT, double n0) {
    g.nx = nx; g.ny = ny; g.nz = nz;
    g.N = (long long)nx * ny * nz;
    g.lx = lx; g.ly = ly; g.lz = lz;
    g.dx = lx / nx; g.dy = ly / ny; g.dz = lz / nz;
    g.dv = g.dx * g.dy * g.dz;
    g.mmax = mmax; g.mrso = mrso;
    g.ntheta = mmax + 1;
    g.nphi = 2 * mmax + 1;
    g.npsi = 2 * (mmax / mrso) + 1;
    g.no = g.ntheta * g.nphi * g.npsi;
    g.nmu2 = mmax / mrso + 1;
    g.np = 0;
    for (int m = 0; m <= mmax; ++m) g.np += (2 * m + 1) * (m / mrso + 1);
    g.kT = kT;
    g.n0 = n0;
    g.rho0 = n0 / (8.0 * kPi * kPi / mrso);
    std::vector<double> x;
    gauss_legendre(g.ntheta, x, g.wtheta);
    g.theta.resize(g.ntheta);
    for (int i = 0; i < g.ntheta; ++i) g.theta[i] = std::acos(x[i]);
    g.phi.resize(g.nphi);
    g.psi.resize(g.npsi);
    for (int i = 0; i < g.nphi; ++i) g.phi[i] = i * (2.0 * kPi / g.nphi);
    for (int i = 0; i < g.npsi; ++i) g.psi[i] = i * (2.0 * kPi / mrso / g.npsi);
    const double eightpisq = 8.0 * kPi * kPi;
    g.w.resize(g.no);
    g.rotm.resize(9 * (size_t)g.no);
    double wsum = 0;
    for (int it = 0, io = 0; it < g.ntheta; ++it)
        for (int ip = 0; ip < g.nphi; ++ip)
            for (int is = 0; is < g.npsi; ++is, ++io) {
                g.w[io] = g.wtheta[it] * (1.0 / g.nphi) * (1.0 / (g.npsi * mrso)) * eightpisq;
                wsum += g.w[io];
                double ct = std::cos(g.theta[it]), st = std::sin(g.theta[it]);
                double cp = std::cos(g.phi[ip]), sp = std::sin(g.phi[ip]);
                double cs = std::cos(g.psi[is]), ss = std::sin(g.psi[is]);
                double *R = &g.rotm[9 * (size_t)io];
                if (g.no == 1) {
                    const double I3[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
                    std::memcpy(R, I3, sizeof I3);
                } else {
                    R[0] = ct * cp * cs - sp * ss;  R[1] = -ct * cp * ss - sp * cs; R[2] = st * cp;
                    R[3] = ct * sp * cs + cp * ss;  R[4] = -ct * sp * ss + cp * cs; R[5] = st * sp;
                    R[6] = -st * cs;                R[7] = st * ss;                 R[8] = ct;
                }
            }
    if (std::lround(std::fabs(wsum / (eightpisq / mrso))) != 1) {
        set_error("angular quadrature does not sum to 8 pi^2/mrso");
        return -1;
    }
    g.pm.clear(); g.pmup.clear(); g.pmu.clear();
    for (int m = 0; m <= mmax; ++m)
        for (int mup = -m; mup <= m; ++mup)
            for (int mu = 0; mu <= m; mu += mrso) {
                g.pm.push_back(m);
                g.pmup.push_back(mup);
                g.pmu.push_back(mu);
            }
    const double twopi = 2.0 * kPi;  // kproj: src/module_grid.f90:319-331
    auto kproj = [twopi](int n, double L, int l) { return (l <= n / 2 + 1) ? (l - 1) * twopi / L : (l - 1 - n) * twopi / L; };
    g.kx.resize(nx); g.ky.resize(ny); g.kz.resize(nz);
    for (int l = 1; l <= nx; ++l) g.kx[l - 1] = kproj(nx, lx, l);
    for (int l = 1; l <= ny; ++l) g.ky[l - 1] = kproj(ny, ly, l);
    for (int l = 1; l <= nz; ++l) g.kz[l - 1] = kproj(nz, lz, l);
    g.wig.resize((size_t)g.np * g.ntheta);
    for (int p = 0; p < g.np; ++p)
        for (int i = 0; i < g.ntheta; ++i)
            g.wig[(size_t)p * g.ntheta + i] = wigner_small_d(g.pm[p], g.pmup[p], g.pmu[p], g.theta[i]);
    return 0;
}

// Dense angular transforms.
//  project (angl2proj, src/module_orientation_projection_transform.f90:159-199):
//    p(ip) = sum_io o(io) A(io, ip),
//    A = fm(m) wtheta d^m_{mup,mu}(theta) e^{+i(mup phi + mu psi)} / (nphi npsi)
//  gather (proj2angl, :202-243; the c2r uses the mu >= 0 half spectrum):
//    o(io) = sum_ip c(mu) fm(m) d (Re p cos a + Im p sin a), a = mup phi + mu psi,
//    c = 1 for mu = 0 and 2 otherwise.
// Stored as real matrices Aproj[io][2 np] (re, im interleaved) and Bgath[2 np][no].
inline void build_angular_matrices(const Grid &g, std::vector<double> &Aproj, std::vector<double> &Bgath) {
    const int no = g.no, np = g.np;
    Aproj.assign((size_t)no * 2 * np, 0.0);
    Bgath.assign((size_t)2 * np * no, 0.0);
    for (int it = 0, io = 0; it < g.ntheta; ++it)
        for (int jp = 0; jp < g.nphi; ++jp)
            for (int js = 0; js < g.npsi; ++js, ++io)
                for (int ip = 0; ip < np; ++ip) {
                    int m = g.pm[ip], mup = g.pmup[ip], mu2 = g.pmu[ip] / g.mrso;
                    // exact phase reduction: mup*phi_j = 2 pi (k2 j / nphi), k2 = mup mod nphi
                    int k2 = ((mup % g.nphi) + g.nphi) % g.nphi;
                    long long num = (long long)((k2 * jp) % g.nphi) * g.npsi + (long long)((mu2 * js) % g.npsi) * g.nphi;
                    long long den = (long long)g.nphi * g.npsi;
                    double frac = (double)(num % den) / (double)den;
                    double ca = std::cos(2.0 * kPi * frac), sa = std::sin(2.0 * kPi * frac);
                    double d = g.wig[(size_t)ip * g.ntheta + it];
                    double a = fm_of(m) * g.wtheta[it] * d / (double)(g.nphi * g.npsi);
                    Aproj[(size_t)io * 2 * np + 2 * ip + 0] = a * ca;
                    Aproj[(size_t)io * 2 * np + 2 * ip + 1] = a * sa;
                    double b = (mu2 == 0 ? 1.0 : 2.0) * fm_of(m) * d;
                    Bgath[(size_t)(2 * ip + 0) * no + io] = b * ca;
                    Bgath[(size_t)(2 * ip + 1) * no + io] = b * sa;
                }
}

// ------------------------------------------------------------------------
// c(k) tables in Luc's format (src/module_read_c_luc.f90:6-124), the step dq
// of src/module_input.f90:591-650 and the preparation of
// src/module_energy_cproj_mrso.f90:362-431: reorder into (m, khi, mu2, n, nu2)
// with nu2 fastest, conjugate, multiply by (-1)^(khi+nu) if nu<0 else (-1)^n.
struct CTable {
    int ncoef = 0, nq = 0;
    double dq = 0;
    std::vector<double> c;        // [nq][ncoef][2]
    std::vector<int> ia_start;    // first coefficient of each output projection
};

inline int npluc_of(int mmax) {
    static const int t[6] = {1, 6, 75, 252, 877, 2002};
    return (mmax >= 0 && mmax <= 5) ? t[mmax] : -1;
}

inline int read_ctable(const Grid &g, const char *path, CTable &ct) {
    std::ifstream in(path);
    if (!in) {
        set_error("cannot open c(k) file %s", path ? path : "(null)");
        return -1;
    }
    const int M = g.mmax, mrso = g.mrso, K = M / mrso;
    const int npl = npluc_of(M);
    if (npl < 0) {
        set_error("no c(k) layout for mmax=%d", M);
        return -1;
    }
    std::string line;
    for (int i = 0; i < 11; ++i)
        if (!std::getline(in, line)) { set_error("c(k) file: short header"); return -1; }
    std::vector<std::vector<int>> idx(5, std::vector<int>(npl));
    for (int r = 0; r < 5; ++r) {
        if (!std::getline(in, line)) { set_error("c(k) file: missing index row %d", r); return -1; }
        std::istringstream ss(line);
        std::string label;
        ss >> label;
        for (int j = 0; j < npl; ++j)
            if (!(ss >> idx[r][j])) { set_error("c(k) file: index row %d has fewer than %d entries", r, npl); return -1; }
    }
    std::getline(in, line);  // blank separator
    // qmax from the largest kx, ky and kz(1:nz/2+1) (src/module_energy_cproj_mrso.f90:366)
    const double twopi = 2.0 * kPi;
    auto kmax_of = [twopi](int n, double L) { return (n / 2) * twopi / L; };  // kproj, src/module_grid.f90:319-331
    double qx = kmax_of(g.nx, g.lx), qy = kmax_of(g.ny, g.ly), qz = kmax_of(g.nz, g.lz);
    double qmax = std::sqrt(qx * qx + qy * qy + qz * qz);
    std::vector<double> rows;  // [row][1 + 2 npl]
    const int rw = 1 + 2 * npl;
    std::vector<double> vals(rw);
    size_t nrows = 0;
    while (std::getline(in, line)) {
        for (char &ch : line)
            if (ch == '(' || ch == ')' || ch == ',') ch = ' ';
        const char *p = line.c_str();
        char *end = nullptr;
        int n = 0;
        while (n < rw) {
            double v = std::strtod(p, &end);
            if (end == p) break;
            vals[n++] = v;
            p = end;
        }
        if (n == 0) continue;
        if (n < rw) { set_error("c(k) file: data row %zu has %d numbers, expected %d", nrows + 1, n, rw); return -1; }
        rows.insert(rows.end(), vals.begin(), vals.end());
        ++nrows;
    }
    if (nrows < 4) { set_error("c(k) file: fewer than 4 data rows"); return -1; }
    double dq = rows[3 * rw] - rows[2 * rw];
    if (!(dq > 0)) { set_error("c(k) file: non-increasing abscissa"); return -1; }
    for (size_t r = 1; r < nrows; ++r)
        if ((rows[r * rw] - rows[(r - 1) * rw] - dq) / dq > 1e-5) { set_error("c(k) file: non uniform abscissa"); return -1; }
    int nq = (int)(qmax / dq + 0.5) + 2;
    if ((size_t)nq > nrows) { set_error("c(k) file: %d rows needed for qmax=%g, %zu available", nq, qmax, nrows); return -1; }
    for (int iq = 0; iq < nq; ++iq)
        if (rows[(size_t)iq * rw] > qmax + 2.0 * dq) { set_error("c(k) file: q beyond qmax+2dq in the rows used"); return -1; }
    // tuple -> column
    const int dm = M + 1, dmu = 2 * K + 1, dk = 2 * M + 1;
    auto key = [&](int m, int n, int mu2, int nu2, int khi) { return (((m * dm + n) * dmu + (mu2 + K)) * dmu + (nu2 + K)) * dk + (khi + M); };
    std::vector<int> col((size_t)dm * dm * dmu * dmu * dk, -1);
    for (int j = 0; j < npl; ++j) {
        int m = idx[0][j], n = idx[1][j], mu = idx[2][j], nu = idx[3][j], khi = idx[4][j];
        if (m < 0 || m > M || n < 0 || n > M || std::abs(mu / mrso) > K || std::abs(nu / mrso) > K || std::abs(khi) > M) continue;
        col[key(m, n, mu / mrso, nu / mrso, khi)] = j;
    }
    ct.ncoef = 0;
    ct.ia_start.clear();
    for (int m = 0; m <= M; ++m)
        for (int khi = -m; khi <= m; ++khi)
            for (int mu2 = 0; mu2 <= m / mrso; ++mu2) {
                ct.ia_start.push_back(ct.ncoef);
                for (int n = std::abs(khi); n <= M; ++n) ct.ncoef += 2 * (n / mrso) + 1;
            }
    ct.nq = nq;
    ct.dq = dq;
    ct.c.assign((size_t)nq * ct.ncoef * 2, 0.0);
    int ia = 0;
    for (int m = 0; m <= M; ++m)
        for (int khi = -m; khi <= m; ++khi)
            for (int mu2 = 0; mu2 <= m / mrso; ++mu2)
                for (int n = std::abs(khi); n <= M; ++n)
                    for (int nu2 = -n / mrso; nu2 <= n / mrso; ++nu2, ++ia) {
                        int j = col[key(m, n, mu2, nu2, khi)];
                        if (j < 0) {
                            set_error("c(k) file lacks (m,n,mu,nu,khi)=(%d,%d,%d,%d,%d)", m, n, mu2 * mrso, nu2 * mrso, khi);
                            return -1;
                        }
                        int nu = nu2 * mrso;
                        double sgn = (nu < 0) ? neg1pow(khi + nu) : neg1pow(n);
                        for (int iq = 0; iq < nq; ++iq) {
                            const double *r = &rows[(size_t)iq * rw];
                            ct.c[((size_t)iq * ct.ncoef + ia) * 2 + 0] = sgn * r[1 + 2 * j];
                            ct.c[((size_t)iq * ct.ncoef + ia) * 2 + 1] = -sgn * r[2 + 2 * j];  // conjugate
                        }
                    }
    return 0;
}

}  // namespace mdft
