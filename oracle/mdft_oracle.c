/*
 * mdft_oracle.c -- FP64 CPU restatement of the MDFT energy-and-gradient path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA engine:
 * only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may
 * load it.  The product library never links, loads or calls it.
 *
 * Parity status: the Fortran reference (dborgis/mdft-dev_general) cannot be
 * compiled on this machine (no Fortran compiler, no FFTW library), so the
 * energy/gradient path is "parity unpinned" against the reference's own
 * outputs; the reference ships no golden energy/gradient vectors.  What is
 * pinned: the Wigner small-d closed forms of
 * tools/test_function_harm_sph_de_luc.f90:23-35, the quadrature normalisation
 * check of src/module_grid.f90:147-154 and the index-map self checks.
 * Every function cites the reference lines it restates.
 *
 * FFTs: FFTW 3.3.4 (vendored as src/fftw-3.3.4.tar.gz, not built here) is
 * replaced by a plain mixed-radix FP64 FFT with the same sign conventions
 * (differences are at the 1e-16 relative level).
 *
 * Array layouts follow the reference (Fortran column major, first index
 * fastest): xi, vext, df are [iz][iy][ix][io] with io fastest.
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double complex cplx;

/* Reductions sum ORC_NCHUNK fixed chunks in order, so results do not depend on
   the number of OpenMP threads. */
#define ORC_NCHUNK 64

#define ORC_PI 3.14159265358979323846264338327950288
static const double EPSDP = 2.220446049250313080847263336181640625e-16; /* epsilon(1._dp) */
static const double EPSSP = 1.1920928955078125e-07;                     /* epsilon(1.)    */

static char g_err[512];
static void set_err(const char *m) { snprintf(g_err, sizeof g_err, "%s", m); }
const char *orc_last_error(void) { return g_err; }

/* ------------------------------------------------------------------------- */
/* factorials: src/module_mathematica.f90:9-44                              */
static double fact(int n)
{
    double r = 1.0;
    for (int i = 2; i <= n; ++i) r *= (double)i;
    return r;
}

static double ipow(double x, int n) /* Fortran real**integer */
{
    double r = 1.0;
    for (int i = 0; i < n; ++i) r *= x;
    return r;
}

/* ------------------------------------------------------------------------- */
/* Wigner small d: src/module_wigner_d.f90:6-60 (argument order m, mu, mup). */
double orc_wigner_small_d(int m, int mu, int mup, double theta)
{
    if (abs(mu) > m || abs(mup) > m) return 0.0;
    if (m == 0) return 1.0;
    if (mu == 0 || mup == 0) {
        int mu0 = mu;
        double theta0 = theta;
        if (mu == 0) { mu0 = mup; theta0 = -theta; }
        double x = 1.0;
        if (mu0 < 0) { x = (mu0 % 2 == 0) ? 1.0 : -1.0; mu0 = -mu0; }
        double cc = cos(theta0), pm1 = 0.0, pm = 1.0, pm2;
        for (int l = mu0 + 1; l <= m; ++l) {
            pm2 = pm1;
            pm1 = pm;
            pm = (cc * (double)(2 * l - 1) * pm1 - (double)(l + mu0 - 1) * pm2) / (double)(l - mu0);
        }
        double sgn = (mu0 % 2 == 0) ? 1.0 : -1.0;
        return x * sgn * sqrt(fact(m - mu0) / fact(m + mu0)) * fact(2 * mu0) /
               (ipow(2.0, mu0) * fact(mu0)) * ipow(sin(theta0), mu0) * pm;
    }
    double d = 0.0, cc = cos(0.5 * theta), ss = sin(0.5 * theta);
    int itmin = (mu - mup > 0) ? mu - mup : 0;
    int itmax = (m + mu < m - mup) ? m + mu : m - mup;
    for (int it = itmin; it <= itmax; ++it) {
        double sgn = (it % 2 == 0) ? 1.0 : -1.0;
        d = d + sgn / (fact(m + mu - it) * fact(m - mup - it) * fact(it) * fact(it - mu + mup)) *
                    ipow(cc, 2 * m + mu - mup - 2 * it) * ipow(ss, 2 * it - mu + mup);
    }
    return sqrt(fact(m + mu) * fact(m - mu) * fact(m + mup) * fact(m - mup)) * d;
}

/* ------------------------------------------------------------------------- */
/* Gauss-Legendre: src/module_grid.f90:262-301 (weights normalised to 1).    */
int orc_gauss_legendre(int n, double *x, double *w)
{
    if (n <= 0) return -1;
    int m = (n + 1) / 2;
    for (int i = 1; i <= m; ++i) {
        double xi = cos(ORC_PI * (i - 0.25) / (n + 0.5));
        double deltaxi = 1.0, p1 = 0, p2 = 0, p3, pp = 0;
        while (fabs(deltaxi) > EPSDP) {
            p1 = 1.0;
            p2 = 0.0;
            for (int j = 1; j <= n; ++j) {
                p3 = p2;
                p2 = p1;
                p1 = ((double)(2 * j - 1) * xi * p2 - (double)(j - 1) * p3) / (double)j;
            }
            pp = n * (xi * p1 - p2) / (xi * xi - 1.0);
            deltaxi = -p1 / pp;
            xi = xi + deltaxi;
        }
        x[i - 1] = xi;
        w[i - 1] = 1.0 / ((1.0 - xi * xi) * pp * pp);
        x[n - i] = -xi;
        w[n - i] = w[i - 1];
    }
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Rotation matrices between complex spherical harmonics:                    */
/* src/module_rotation.f90:13-34 (coefficients) and :119-247 (recursion).    */
#define RMAX 6
static double rot_a[RMAX + 1][2 * RMAX + 1][2 * RMAX + 1], rot_b[RMAX + 1][2 * RMAX + 1][2 * RMAX + 1];
static double rot_c[RMAX + 1][2 * RMAX + 1], rot_d[RMAX + 1][2 * RMAX + 1];
static int rot_ready = 0;

static double sqrtof(int k) { return k <= 0 ? 0.0 : sqrt((double)k); }

static void rotation_init(void)
{
    if (rot_ready) return;
    const double sqrt2 = sqrt(2.0);
    memset(rot_a, 0, sizeof rot_a);
    memset(rot_b, 0, sizeof rot_b);
    memset(rot_c, 0, sizeof rot_c);
    memset(rot_d, 0, sizeof rot_d);
    for (int l = 2; l <= RMAX; ++l)
        for (int m = -l; m <= l; ++m) {
            for (int m1 = -l + 1; m1 <= l - 1; ++m1) {
                rot_a[l][m + RMAX][m1 + RMAX] = sqrtof(l + m) * sqrtof(l - m) / (sqrtof(l + m1) * sqrtof(l - m1));
                rot_b[l][m + RMAX][m1 + RMAX] =
                    sqrtof(l + m) * sqrtof(l + m - 1) / (sqrt2 * sqrtof(l + m1) * sqrtof(l - m1));
            }
            int m1 = l;
            rot_c[l][m + RMAX] = sqrt2 * sqrtof(l + m) * sqrtof(l - m) / (sqrtof(l + m1) * sqrtof(l + m1 - 1));
            rot_d[l][m + RMAX] = sqrtof(l + m) * sqrtof(l + m - 1) / (sqrtof(l + m1) * sqrtof(l + m1 - 1));
        }
    rot_ready = 1;
}

/* R is (mmax+1) x (2mmax+1) x (2mmax+1) complex, index R[(l*(2M+1) + m+M)*(2M+1) + m1+M]. */
#define RIDX(l, m, m1, M) ((((l) * (2 * (M) + 1) + ((m) + (M))) * (2 * (M) + 1)) + ((m1) + (M)))
int orc_rotation_matrix(int mmax, const double q[3], double *Rout /* complex interleaved */)
{
    if (mmax > RMAX || mmax < 0) return -1;
    rotation_init();
    const int M = mmax, W = 2 * mmax + 1;
    const int sz = (mmax + 1) * W * W;
    double *f = calloc(sz, sizeof(double)), *g = calloc(sz, sizeof(double));
    if (mmax == 0) {
        for (int i = 0; i < sz; ++i) { Rout[2 * i] = 1.0; Rout[2 * i + 1] = 0.0; }
        free(f); free(g);
        return 0;
    }
    const double sqrt2 = sqrt(2.0);
    double r3[3], r2[3], r1[3];
    f[RIDX(0, 0, 0, M)] = 1.0;
    if (q[0] == 0.0 && q[1] == 0.0 && q[2] == 0.0) { r3[0] = 0; r3[1] = 0; r3[2] = 1; }
    else { r3[0] = q[0]; r3[1] = q[1]; r3[2] = q[2]; }
    if (r3[0] != 0.0 || r3[1] != 0.0) { /* cross((0,0,1), r3) */
        r2[0] = 0.0 * r3[2] - 1.0 * r3[1];
        r2[1] = 1.0 * r3[0] - 0.0 * r3[2];
        r2[2] = 0.0 * r3[1] - 0.0 * r3[0];
    } else { /* cross(r3, (1,0,0)) */
        r2[0] = r3[1] * 0.0 - r3[2] * 0.0;
        r2[1] = r3[2] * 1.0 - r3[0] * 0.0;
        r2[2] = r3[0] * 0.0 - r3[1] * 1.0;
    }
    double n3 = sqrt(r3[0] * r3[0] + r3[1] * r3[1] + r3[2] * r3[2]);
    double n2 = sqrt(r2[0] * r2[0] + r2[1] * r2[1] + r2[2] * r2[2]);
    for (int i = 0; i < 3; ++i) { r3[i] /= n3; r2[i] /= n2; }
    r1[0] = r2[1] * r3[2] - r2[2] * r3[1];
    r1[1] = r2[2] * r3[0] - r2[0] * r3[2];
    r1[2] = r2[0] * r3[1] - r2[1] * r3[0];
    /* rmat(i,j): column j is r_j; rmat(i,j) = r_j[i] */
#define RM(i, j) ((j) == 1 ? r1[(i)-1] : ((j) == 2 ? r2[(i)-1] : r3[(i)-1]))
#define F(l, m, m1) f[RIDX(l, m, m1, M)]
#define G(l, m, m1) g[RIDX(l, m, m1, M)]
    F(1, -1, -1) = (RM(2, 2) + RM(1, 1)) * 0.5;
    F(1, -1, 0) = RM(1, 3) / sqrt2;
    F(1, -1, 1) = (RM(2, 2) - RM(1, 1)) * 0.5;
    F(1, 0, -1) = RM(3, 1) / sqrt2;
    F(1, 0, 0) = RM(3, 3);
    F(1, 0, 1) = -RM(3, 1) / sqrt2;
    F(1, 1, -1) = (RM(2, 2) - RM(1, 1)) * 0.5;
    F(1, 1, 0) = -RM(1, 3) / sqrt2;
    F(1, 1, 1) = (RM(2, 2) + RM(1, 1)) * 0.5;
    G(1, -1, -1) = (RM(2, 1) - RM(1, 2)) * 0.5;
    G(1, -1, 0) = RM(2, 3) / sqrt2;
    G(1, -1, 1) = (-RM(2, 1) - RM(1, 2)) * 0.5;
    G(1, 0, -1) = -RM(3, 2) / sqrt2;
    G(1, 0, 0) = 0.0;
    G(1, 0, 1) = -RM(3, 2) / sqrt2;
    G(1, 1, -1) = (RM(2, 1) + RM(1, 2)) * 0.5;
    G(1, 1, 0) = RM(2, 3) / sqrt2;
    G(1, 1, 1) = (RM(1, 2) - RM(2, 1)) * 0.5;
#define A(l, m, m1) rot_a[l][(m) + RMAX][(m1) + RMAX]
#define B(l, m, m1) rot_b[l][(m) + RMAX][(m1) + RMAX]
#define C(l, m) rot_c[l][(m) + RMAX]
#define D(l, m) rot_d[l][(m) + RMAX]
    for (int l = 2; l <= mmax; ++l) {
        int l1 = l - 1;
        for (int m = -l; m <= l; ++m) {
            int m1min = (m > 0) ? 1 : 0;
            for (int m1 = m1min; m1 <= l - 1; ++m1) {
                if (m == -l) {
                    F(l, m, m1) = B(l, -m, m1) * (F(1, -1, 0) * F(l1, m + 1, m1) - G(1, -1, 0) * G(l1, m + 1, m1));
                    G(l, m, m1) = B(l, -m, m1) * (F(1, -1, 0) * G(l1, m + 1, m1) + G(1, -1, 0) * F(l1, m + 1, m1));
                } else if (m == l) {
                    F(l, m, m1) = B(l, m, m1) * (F(1, 1, 0) * F(l1, m - 1, m1) - G(1, 1, 0) * G(l1, m - 1, m1));
                    G(l, m, m1) = B(l, m, m1) * (F(1, 1, 0) * G(l1, m - 1, m1) + G(1, 1, 0) * F(l1, m - 1, m1));
                } else {
                    F(l, m, m1) = A(l, m, m1) * (F(1, 0, 0) * F(l1, m, m1)) +
                                  B(l, m, m1) * (F(1, 1, 0) * F(l1, m - 1, m1) - G(1, 1, 0) * G(l1, m - 1, m1)) +
                                  B(l, -m, m1) * (F(1, -1, 0) * F(l1, m + 1, m1) - G(1, -1, 0) * G(l1, m + 1, m1));
                    G(l, m, m1) = A(l, m, m1) * (F(1, 0, 0) * G(l1, m, m1)) +
                                  B(l, m, m1) * (F(1, 1, 0) * G(l1, m - 1, m1) + G(1, 1, 0) * F(l1, m - 1, m1)) +
                                  B(l, -m, m1) * (F(1, -1, 0) * G(l1, m + 1, m1) + G(1, -1, 0) * F(l1, m + 1, m1));
                }
                double s = ((m + m1) % 2 == 0) ? 1.0 : -1.0;
                F(l, -m, -m1) = s * F(l, m, m1);
                G(l, -m, -m1) = -s * G(l, m, m1);
            }
            int m1 = l;
            if (m == -l) {
                F(l, m, m1) = D(l, -m) * (F(1, -1, 1) * F(l1, m + 1, m1 - 1) - G(1, -1, 1) * G(l1, m + 1, m1 - 1));
                G(l, m, m1) = D(l, -m) * (F(1, -1, 1) * G(l1, m + 1, m1 - 1) + G(1, -1, 1) * F(l1, m + 1, m1 - 1));
            } else if (m == l) {
                F(l, m, m1) = D(l, m) * (F(1, 1, 1) * F(l1, m - 1, m1 - 1) - G(1, 1, 1) * G(l1, m - 1, m1 - 1));
                G(l, m, m1) = D(l, m) * (F(1, 1, 1) * G(l1, m - 1, m1 - 1) + G(1, 1, 1) * F(l1, m - 1, m1 - 1));
            } else {
                F(l, m, m1) = C(l, m) * (F(1, 0, 1) * F(l1, m, m1 - 1) - G(1, 0, 1) * G(l1, m, m1 - 1)) +
                              D(l, m) * (F(1, 1, 1) * F(l1, m - 1, m1 - 1) - G(1, 1, 1) * G(l1, m - 1, m1 - 1)) +
                              D(l, -m) * (F(1, -1, 1) * F(l1, m + 1, m1 - 1) - G(1, -1, 1) * G(l1, m + 1, m1 - 1));
                G(l, m, m1) = C(l, m) * (F(1, 0, 1) * G(l1, m, m1 - 1) + G(1, 0, 1) * F(l1, m, m1 - 1)) +
                              D(l, m) * (F(1, 1, 1) * G(l1, m - 1, m1 - 1) + G(1, 1, 1) * F(l1, m - 1, m1 - 1)) +
                              D(l, -m) * (F(1, -1, 1) * G(l1, m + 1, m1 - 1) + G(1, -1, 1) * F(l1, m + 1, m1 - 1));
            }
            double s = ((m + m1) % 2 == 0) ? 1.0 : -1.0;
            F(l, -m, -m1) = s * F(l, m, m1);
            G(l, -m, -m1) = -s * G(l, m, m1);
        }
    }
    for (int i = 0; i < sz; ++i) { Rout[2 * i] = f[i]; Rout[2 * i + 1] = g[i]; }
    free(f);
    free(g);
    return 0;
#undef RM
#undef F
#undef G
#undef A
#undef B
#undef C
#undef D
}

/* ------------------------------------------------------------------------- */
/* Plain FP64 FFT (stand-in for FFTW): X[k] = sum_j x[j] exp(sign*2*pi*i*j*k/n) */
static void fft1d_rec(cplx *x, int n, int stride, cplx *out, int sign, cplx *scratch)
{
    if (n == 1) { out[0] = x[0]; return; }
    int r = 0;
    if (n % 4 == 0) r = 4;
    else if (n % 2 == 0) r = 2;
    else if (n % 3 == 0) r = 3;
    else if (n % 5 == 0) r = 5;
    if (r == 0) { /* direct DFT for other primes */
        for (int k = 0; k < n; ++k) {
            cplx s = 0;
            for (int j = 0; j < n; ++j) {
                double ang = sign * 2.0 * ORC_PI * (double)((long)j * k % n) / n;
                s += x[j * stride] * (cos(ang) + I * sin(ang));
            }
            out[k] = s;
        }
        return;
    }
    int m = n / r;
    /* sub-transforms of decimated sequences into scratch */
    for (int q = 0; q < r; ++q) fft1d_rec(x + q * stride, m, stride * r, scratch + q * m, sign, out);
    for (int k = 0; k < m; ++k) {
        cplx t[5];
        for (int q = 0; q < r; ++q) {
            double ang = sign * 2.0 * ORC_PI * (double)(q * k) / n;
            t[q] = scratch[q * m + k] * (cos(ang) + I * sin(ang));
        }
        for (int s = 0; s < r; ++s) {
            cplx acc = 0;
            for (int q = 0; q < r; ++q) {
                double ang = sign * 2.0 * ORC_PI * (double)((q * s) % r) / r;
                acc += t[q] * (cos(ang) + I * sin(ang));
            }
            out[k + s * m] = acc;
        }
    }
}

static void fft1d(cplx *x, int n, int sign)
{
    cplx *out = malloc(sizeof(cplx) * n), *scr = malloc(sizeof(cplx) * n);
    fft1d_rec(x, n, 1, out, sign, scr);
    memcpy(x, out, sizeof(cplx) * n);
    free(out);
    free(scr);
}

/* 3-D in-place c2c on a[(iz*ny+iy)*nx+ix] */
static void fft3d(cplx *a, int nx, int ny, int nz, int sign)
{
#pragma omp parallel
    {
        int nm = nx > ny ? nx : ny;
        nm = nm > nz ? nm : nz;
        cplx *line = malloc(sizeof(cplx) * nm);
#pragma omp for collapse(2)
        for (int iz = 0; iz < nz; ++iz)
            for (int iy = 0; iy < ny; ++iy) fft1d(a + ((long)iz * ny + iy) * nx, nx, sign);
#pragma omp for collapse(2)
        for (int iz = 0; iz < nz; ++iz)
            for (int ix = 0; ix < nx; ++ix) {
                for (int iy = 0; iy < ny; ++iy) line[iy] = a[((long)iz * ny + iy) * nx + ix];
                fft1d(line, ny, sign);
                for (int iy = 0; iy < ny; ++iy) a[((long)iz * ny + iy) * nx + ix] = line[iy];
            }
#pragma omp for collapse(2)
        for (int iy = 0; iy < ny; ++iy)
            for (int ix = 0; ix < nx; ++ix) {
                for (int iz = 0; iz < nz; ++iz) line[iz] = a[((long)iz * ny + iy) * nx + ix];
                fft1d(line, nz, sign);
                for (int iz = 0; iz < nz; ++iz) a[((long)iz * ny + iy) * nx + ix] = line[iz];
            }
        free(line);
    }
}

/* ------------------------------------------------------------------------- */
/* The evaluation context (grid, quadrature, tables, c(k), vext).            */
typedef struct orc {
    int nx, ny, nz;
    long N;
    double lx, ly, lz, dx, dy, dz, dv;
    int mmax, mrso, ntheta, nphi, npsi, no, np, nmu2;
    double *thetaof, *wthetaof, *phiof, *psiof, *w; /* w[no] */
    double *kx, *ky, *kz;
    double *rotm;                /* [no][9] row major rot(io) */
    int *p3m, *p3mup, *p3mu;     /* [np] */
    int *p3p;                    /* [(m)(2M+1)(nmu2)] -> ip (0-based) or -1 */
    double *wig;                 /* [np][ntheta] */
    cplx *ef, *eb;               /* DFT phases [nmu2][nphi][nphi*npsi], sign -1 / +1 */
    double kT, n0, rho0;
    /* prepared c table */
    int ncoef, nq;
    double dq;
    cplx *c; /* [nq][ncoef] */
    double *vext; /* [N][no], owned */
    double const_corr; /* charged-solute corrections added to F (constant in xi) */
    /* bridge = "cgb" (0: none, 1: 'sla', 2: 'wda') and its parameters */
    int cgb;
    double cgb_B6, cgb_sigma, cgb_c00;
    /* bridge = "hard_sphere" (0: none, 1: PY, 2: CS): radius, bulk excess chemical potential
       and grand potential, and the hard-sphere c(k) on nb_k points of step dq */
    int fmt;
    double hs_R, hs_mu, hs_fexc0;
    int hs_nbk;
    double *hs_cs;
    cplx *drho; /* [N][np] */
} orc;

static const double fm_tab[8] = {1.0, 1.7320508075688772, 2.23606797749979, 2.6457513110645907,
                                 3.0, 3.3166247903554, 3.605551275463989, 3.7416573867739413};
/* fm(0:7) = sqrt(2m+1) except fm(7)=sqrt(14): module_orientation_projection_transform.f90:35 */

static inline int p3idx(const orc *o, int m, int mup, int mu2)
{
    return (m * (2 * o->mmax + 1) + (mup + o->mmax)) * o->nmu2 + mu2;
}

/* module_grid.f90:319-331 */
static double kproj(int n, double len, int l /*1-based*/)
{
    const double twopi = 2.0 * ORC_PI;
    if (l <= n / 2 + 1) return (l - 1) * twopi / len;
    return (l - 1 - n) * twopi / len;
}

void orc_destroy(orc *o)
{
    if (!o) return;
    free(o->thetaof); free(o->wthetaof); free(o->phiof); free(o->psiof); free(o->w);
    free(o->kx); free(o->ky); free(o->kz); free(o->rotm);
    free(o->p3m); free(o->p3mup); free(o->p3mu); free(o->p3p); free(o->wig); free(o->ef); free(o->eb);
    free(o->c); free(o->vext); free(o->drho); free(o->hs_cs);
    free(o);
}

/* module_grid.f90:51-212 + module_energy_cproj_mrso.f90:151-235 tables */
orc *orc_create(int nx, int ny, int nz, double lx, double ly, double lz, int mmax, int mrso, double kT, double n0)
{
    if (nx <= 0 || ny <= 0 || nz <= 0 || mmax < 0 || mmax > 6 || mrso <= 0) { set_err("bad grid"); return NULL; }
    orc *o = calloc(1, sizeof(orc));
    o->nx = nx; o->ny = ny; o->nz = nz; o->N = (long)nx * ny * nz;
    o->lx = lx; o->ly = ly; o->lz = lz;
    o->dx = lx / nx; o->dy = ly / ny; o->dz = lz / nz;
    o->dv = o->dx * o->dy * o->dz;
    o->mmax = mmax; o->mrso = mrso;
    o->ntheta = mmax + 1; o->nphi = 2 * mmax + 1; o->npsi = 2 * (mmax / mrso) + 1;
    o->no = o->ntheta * o->nphi * o->npsi;
    o->nmu2 = mmax / mrso + 1;
    int np = 0;
    for (int m = 0; m <= mmax; ++m) np += (2 * m + 1) * (m / mrso + 1);
    o->np = np;
    o->kT = kT; o->n0 = n0;
    o->rho0 = n0 / (8.0 * ORC_PI * ORC_PI / mrso); /* module_solvent.f90:222 */
    const double twopi = 2.0 * ORC_PI, eightpisq = 8.0 * ORC_PI * ORC_PI;
    double dphi = twopi / (double)o->nphi;
    double dpsi = twopi / (double)mrso / (double)o->npsi;
    o->thetaof = malloc(sizeof(double) * o->ntheta);
    o->wthetaof = malloc(sizeof(double) * o->ntheta);
    o->phiof = malloc(sizeof(double) * o->nphi);
    o->psiof = malloc(sizeof(double) * o->npsi);
    o->w = malloc(sizeof(double) * o->no);
    o->rotm = malloc(sizeof(double) * 9 * o->no);
    for (int i = 0; i < o->npsi; ++i) o->psiof[i] = (double)i * dpsi;
    for (int i = 0; i < o->nphi; ++i) o->phiof[i] = (double)i * dphi;
    orc_gauss_legendre(o->ntheta, o->thetaof, o->wthetaof);
    for (int i = 0; i < o->ntheta; ++i) o->thetaof[i] = acos(o->thetaof[i]);
    double wphi = 1.0 / (double)o->nphi, wpsi = 1.0 / (double)(o->npsi * mrso);
    int io = 0;
    double wsum = 0;
    for (int it = 0; it < o->ntheta; ++it)
        for (int ip = 0; ip < o->nphi; ++ip)
            for (int is = 0; is < o->npsi; ++is, ++io) {
                o->w[io] = o->wthetaof[it] * wphi * wpsi * eightpisq;
                wsum += o->w[io];
                double th = o->thetaof[it], ph = o->phiof[ip], ps = o->psiof[is];
                double ct = cos(th), st = sin(th), cp = cos(ph), sp = sin(ph), cs = cos(ps), ss = sin(ps);
                double *R = o->rotm + 9 * io;
                if (o->no == 1) {
                    R[0] = 1; R[1] = 0; R[2] = 0; R[3] = 0; R[4] = 1; R[5] = 0; R[6] = 0; R[7] = 0; R[8] = 1;
                } else { /* module_grid.f90:187-206 */
                    R[0] = ct * cp * cs - sp * ss;
                    R[1] = -ct * cp * ss - sp * cs;
                    R[2] = st * cp;
                    R[3] = ct * sp * cs + cp * ss;
                    R[4] = -ct * sp * ss + cp * cs;
                    R[5] = st * sp;
                    R[6] = -st * cs;
                    R[7] = st * ss;
                    R[8] = ct;
                }
            }
    /* module_grid.f90:147-154 normalisation self-check */
    if (lround(fabs(wsum / (eightpisq / mrso))) != 1) { set_err("quadrature normalisation check failed"); orc_destroy(o); return NULL; }
    o->kx = malloc(sizeof(double) * nx);
    o->ky = malloc(sizeof(double) * ny);
    o->kz = malloc(sizeof(double) * nz);
    for (int l = 1; l <= nx; ++l) o->kx[l - 1] = kproj(nx, lx, l);
    for (int l = 1; l <= ny; ++l) o->ky[l - 1] = kproj(ny, ly, l);
    for (int l = 1; l <= nz; ++l) o->kz[l - 1] = kproj(nz, lz, l);
    /* projection index maps: module_orientation_projection_transform.f90:80-101 */
    o->p3m = malloc(sizeof(int) * np);
    o->p3mup = malloc(sizeof(int) * np);
    o->p3mu = malloc(sizeof(int) * np);
    int np3 = (mmax + 1) * (2 * mmax + 1) * o->nmu2;
    o->p3p = malloc(sizeof(int) * np3);
    for (int i = 0; i < np3; ++i) o->p3p[i] = -1;
    int ip = 0;
    for (int m = 0; m <= mmax; ++m)
        for (int mup = -m; mup <= m; ++mup)
            for (int mu = 0; mu <= m; mu += mrso) {
                o->p3p[p3idx(o, m, mup, mu / mrso)] = ip;
                o->p3m[ip] = m; o->p3mup[ip] = mup; o->p3mu[ip] = mu;
                ++ip;
            }
    if (ip != np) { set_err("ip /= np"); orc_destroy(o); return NULL; }
    /* Wigner table: module_orientation_projection_transform.f90:124-133 */
    o->wig = malloc(sizeof(double) * np * o->ntheta);
    for (int p = 0; p < np; ++p)
        for (int i = 0; i < o->ntheta; ++i)
            o->wig[p * o->ntheta + i] = orc_wigner_small_d(o->p3m[p], o->p3mup[p], o->p3mu[p], o->thetaof[i]);
    {
        const int nphi = o->nphi, npsi = o->npsi, nmu2 = o->nmu2;
        o->ef = malloc(sizeof(cplx) * nmu2 * nphi * nphi * npsi);
        o->eb = malloc(sizeof(cplx) * nmu2 * nphi * nphi * npsi);
        for (int k1 = 0; k1 < nmu2; ++k1)
            for (int k2 = 0; k2 < nphi; ++k2)
                for (int j2 = 0; j2 < nphi; ++j2)
                    for (int j1 = 0; j1 < npsi; ++j1) {
                        double ang = 2.0 * ORC_PI * ((double)((k1 * j1) % npsi) / npsi + (double)((k2 * j2) % nphi) / nphi);
                        size_t id = ((size_t)(k1 * nphi + k2) * nphi + j2) * npsi + j1;
                        o->ef[id] = cos(ang) - I * sin(ang);
                        o->eb[id] = cos(ang) + I * sin(ang);
                    }
    }
    o->vext = calloc((size_t)o->N * o->no, sizeof(double));
    o->drho = malloc(sizeof(cplx) * (size_t)o->N * np);
    return o;
}

int orc_dims(const orc *o, int *out /* ntheta nphi npsi no np ncoef nq */)
{
    out[0] = o->ntheta; out[1] = o->nphi; out[2] = o->npsi; out[3] = o->no; out[4] = o->np;
    out[5] = o->ncoef; out[6] = o->nq;
    return 0;
}
int orc_weights(const orc *o, double *w) { memcpy(w, o->w, sizeof(double) * o->no); return 0; }
int orc_rotm(const orc *o, double *r) { memcpy(r, o->rotm, sizeof(double) * 9 * o->no); return 0; }
double orc_rho0(const orc *o) { return o->rho0; }
double orc_dv(const orc *o) { return o->dv; }
double orc_dq(const orc *o) { return o->dq; }
int orc_set_vext(orc *o, const double *v) { memcpy(o->vext, v, sizeof(double) * o->N * o->no); return 0; }
int orc_get_vext(const orc *o, double *v) { memcpy(v, o->vext, sizeof(double) * o->N * o->no); return 0; }
void orc_set_const_corr(orc *o, double c) { o->const_corr = c; }
int orc_ctable(const orc *o, double *out) { memcpy(out, o->c, sizeof(cplx) * (size_t)o->nq * o->ncoef); return 0; }

/* ------------------------------------------------------------------------- */
/* c(k) file reader (module_read_c_luc.f90:6-124; dq from module_input.f90:  */
/* 591-650) and preparation (module_energy_cproj_mrso.f90:362-431).          */
static int npluc_of(int mmax)
{
    static const int t[7] = {1, 6, 75, 252, 877, 2002, -1};
    return t[mmax];
}

static int parse_doubles(char *line, double *out, int maxn)
{
    for (char *p = line; *p; ++p)
        if (*p == '(' || *p == ')' || *p == ',') *p = ' ';
    int n = 0;
    char *p = line, *end;
    while (n < maxn) {
        double v = strtod(p, &end);
        if (end == p) break;
        out[n++] = v;
        p = end;
    }
    return n;
}

int orc_load_ck(orc *o, const char *path)
{
    FILE *fp = fopen(path, "r");
    if (!fp) { set_err("cannot open c(k) file"); return -1; }
    const int mmax = o->mmax, mrso = o->mrso;
    int npl = npluc_of(mmax);
    if (npl < 0) { fclose(fp); set_err("no npluc for this mmax"); return -1; }
    size_t cap = 1 << 23; /* mmax 5 rows are ~100 KB of text */
    char *line = malloc(cap);
    int lineno = 0;
    int *idx[5];
    for (int k = 0; k < 5; ++k) idx[k] = malloc(sizeof(int) * npl);
    double *buf = malloc(sizeof(double) * (2 * npl + 8));
    /* header: 10 comment lines, 'alpha' line, 5 index rows, a blank line */
    while (lineno < 11) {
        if (!fgets(line, cap, fp)) { set_err("short c(k) header"); goto fail; }
        ++lineno;
    }
    for (int k = 0; k < 5; ++k) {
        if (!fgets(line, cap, fp)) { set_err("short c(k) index rows"); goto fail; }
        ++lineno;
        char *p = line;
        while (*p == ' ' || *p == '\t') ++p;
        while (*p && *p != ' ' && *p != '\t') ++p; /* skip label */
        for (int j = 0; j < npl; ++j) {
            char *end;
            long v = strtol(p, &end, 10);
            if (end == p) { set_err("bad c(k) index row"); goto fail; }
            idx[k][j] = (int)v;
            p = end;
        }
    }
    if (!fgets(line, cap, fp)) { set_err("short c(k) file"); goto fail; }
    /* qmax: module_energy_cproj_mrso.f90:366 */
    double mkx = o->kx[0], mky = o->ky[0], mkz = o->kz[0];
    for (int i = 0; i < o->nx; ++i) if (o->kx[i] > mkx) mkx = o->kx[i];
    for (int i = 0; i < o->ny; ++i) if (o->ky[i] > mky) mky = o->ky[i];
    for (int i = 0; i < o->nz / 2 + 1; ++i) if (o->kz[i] > mkz) mkz = o->kz[i];
    double qmax = sqrt(mkx * mkx + mky * mky + mkz * mkz);
    /* read data rows */
    size_t rcap = 1024, nrows = 0;
    double *rows = malloc(sizeof(double) * rcap * (2 * npl + 1));
    while (fgets(line, cap, fp)) {
        int n = parse_doubles(line, buf, 2 * npl + 1);
        if (n == 0) continue;
        if (n < 2 * npl + 1) { set_err("short c(k) data row"); free(rows); goto fail; }
        if (nrows == rcap) { rcap *= 2; rows = realloc(rows, sizeof(double) * rcap * (2 * npl + 1)); }
        memcpy(rows + nrows * (2 * npl + 1), buf, sizeof(double) * (2 * npl + 1));
        ++nrows;
    }
    if (nrows < 4) { set_err("too few c(k) rows"); free(rows); goto fail; }
    double dq = rows[3 * (2 * npl + 1)] - rows[2 * (2 * npl + 1)];
    /* uniform abscissa check (module_input.f90:638-646) */
    for (size_t r = 1; r < nrows; ++r) {
        double d = rows[r * (2 * npl + 1)] - rows[(r - 1) * (2 * npl + 1)];
        if ((d - dq) / dq > 1e-5) { set_err("non uniform abscissa in c(k) file"); free(rows); goto fail; }
    }
    int nq = (int)(qmax / dq + 0.5) + 2;
    if ((size_t)nq > nrows) { set_err("more q values wanted than available in c(k) file"); free(rows); goto fail; }
    for (int iq = 0; iq < nq; ++iq)
        if (rows[iq * (2 * npl + 1)] > qmax + 2.0 * dq) { set_err("q>qmaxwanted"); free(rows); goto fail; }
    /* Luc index map p(m,n,mu2,nu2,khi) */
    int M = mmax, K = mmax / mrso;
    int dm = M + 1, dmu = 2 * K + 1, dkhi = 2 * M + 1;
#define LUCP(m, n, mu2, nu2, khi) (((((m) * dm + (n)) * dmu + ((mu2) + K)) * dmu + ((nu2) + K)) * dkhi + ((khi) + M))
    int *lp = malloc(sizeof(int) * dm * dm * dmu * dmu * dkhi);
    for (int i = 0; i < dm * dm * dmu * dmu * dkhi; ++i) lp[i] = -1;
    for (int j = 0; j < npl; ++j) {
        int m = idx[0][j], n = idx[1][j], mu = idx[2][j], nu = idx[3][j], khi = idx[4][j];
        if (m < 0 || m > M || n < 0 || n > M || abs(mu / mrso) > K || abs(nu / mrso) > K || abs(khi) > M) continue;
        lp[LUCP(m, n, mu / mrso, nu / mrso, khi)] = j;
    }
    /* reorder into (m, khi, mu2, n, nu2) with nu2 fastest */
    int ncoef = 0;
    for (int m = 0; m <= M; ++m)
        for (int khi = -m; khi <= m; ++khi)
            for (int mu2 = 0; mu2 <= m / mrso; ++mu2)
                for (int n = abs(khi); n <= M; ++n)
                    for (int nu2 = -n / mrso; nu2 <= n / mrso; ++nu2) ++ncoef;
    o->ncoef = ncoef; o->nq = nq; o->dq = dq;
    free(o->c);
    o->c = malloc(sizeof(cplx) * (size_t)nq * ncoef);
    int ia = 0;
    for (int m = 0; m <= M; ++m)
        for (int khi = -m; khi <= m; ++khi)
            for (int mu2 = 0; mu2 <= m / mrso; ++mu2)
                for (int n = abs(khi); n <= M; ++n)
                    for (int nu2 = -n / mrso; nu2 <= n / mrso; ++nu2, ++ia) {
                        int j = lp[LUCP(m, n, mu2, nu2, khi)];
                        if (j < 0) { set_err("c(k) file lacks a needed (m,n,mu,nu,khi) tuple"); free(lp); free(rows); goto fail; }
                        int nu = nu2 * mrso;
                        /* sign prefactor: (-1)^(khi+nu) if nu<0 else (-1)^n  (:420-429) */
                        double sgn = (nu < 0) ? (((khi + nu) % 2 == 0) ? 1.0 : -1.0) : ((n % 2 == 0) ? 1.0 : -1.0);
                        for (int iq = 0; iq < nq; ++iq) {
                            const double *rw = rows + iq * (2 * npl + 1);
                            cplx v = rw[1 + 2 * j] + I * rw[2 + 2 * j];
                            o->c[(size_t)iq * ncoef + ia] = sgn * conj(v); /* conj: :415 */
                        }
                    }
#undef LUCP
    free(lp);
    free(rows);
    for (int k = 0; k < 5; ++k) free(idx[k]);
    free(buf);
    free(line);
    fclose(fp);
    return 0;
fail:
    for (int k = 0; k < 5; ++k) free(idx[k]);
    free(buf);
    free(line);
    fclose(fp);
    return -1;
}

/* ------------------------------------------------------------------------- */
/* angl2proj / proj2angl for one grid point:                                 */
/* module_orientation_projection_transform.f90:159-199 and :202-243.         */
static void angl2proj_pt(const orc *o, const double *ov, cplx *p, cplx *ftab /* ntheta*nmu2*(2M+1) */)
{
    const int nth = o->ntheta, nphi = o->nphi, npsi = o->npsi, M = o->mmax, nmu2 = o->nmu2;
    /* f(itheta, mu2, mup) */
#define FT(it, mu2, mup) ftab[((it) * nmu2 + (mu2)) * (2 * M + 1) + ((mup) + M)]
    for (int it = 0; it < nth; ++it) {
        const double *r = ov + it * nphi * npsi; /* r(ipsi, iphi), ipsi fastest */
        for (int k1 = 0; k1 < nmu2; ++k1)
            for (int k2 = 0; k2 < nphi; ++k2) {
                /* r2c with FFTW sign -1: sum r(j1,j2) exp(-2 pi i (k1 j1/npsi + k2 j2/nphi)) */
                cplx s = 0;
                const cplx *e = o->ef + (size_t)(k1 * nphi + k2) * nphi * npsi;
                for (int j2 = 0; j2 < nphi; ++j2)
                    for (int j1 = 0; j1 < npsi; ++j1) s += r[j2 * npsi + j1] * e[j2 * npsi + j1];
                s = conj(s) / (double)(nphi * npsi);
                int mup = (k2 <= M) ? k2 : k2 - nphi; /* :186-187 */
                FT(it, k1, mup) = s;
            }
    }
    int ip = 0;
    for (int m = 0; m <= M; ++m)
        for (int mup = -m; mup <= m; ++mup)
            for (int mu2 = 0; mu2 <= m / o->mrso; ++mu2, ++ip) {
                cplx s = 0;
                for (int it = 0; it < nth; ++it) s += FT(it, mu2, mup) * o->wig[ip * nth + it] * o->wthetaof[it];
                p[ip] = s * fm_tab[m];
            }
#undef FT
}

static void proj2angl_pt(const orc *o, const cplx *p, double *ov, cplx *ftab)
{
    const int nth = o->ntheta, nphi = o->nphi, npsi = o->npsi, M = o->mmax, nmu2 = o->nmu2, mrso = o->mrso;
#define FT(it, mu2, mup) ftab[((it) * nmu2 + (mu2)) * (2 * M + 1) + ((mup) + M)]
    for (int i = 0; i < nth * nmu2 * (2 * M + 1); ++i) ftab[i] = 0;
    for (int mup = -M; mup <= M; ++mup)
        for (int mu2 = 0; mu2 <= M / mrso; ++mu2) {
            int m0 = abs(mup) > mrso * mu2 ? abs(mup) : mrso * mu2;
            for (int m = m0; m <= M; ++m) {
                int ip = o->p3p[p3idx(o, m, mup, mu2)];
                for (int it = 0; it < nth; ++it) FT(it, mu2, mup) += p[ip] * o->wig[ip * nth + it] * fm_tab[m];
            }
        }
    /* c2r (sign +1, un-normalised) of conj(f) over the half spectrum along psi */
    for (int it = 0; it < nth; ++it)
        for (int j2 = 0; j2 < nphi; ++j2)
            for (int j1 = 0; j1 < npsi; ++j1) {
                double acc0 = 0, acc1 = 0;
                for (int k2 = 0; k2 < nphi; ++k2) {
                    int mup = (k2 <= M) ? k2 : k2 - nphi;
                    cplx X = conj(FT(it, 0, mup));
                    acc0 += creal(X * o->eb[((size_t)(0 * nphi + k2) * nphi + j2) * npsi + j1]);
                    for (int k1 = 1; k1 < nmu2; ++k1) {
                        cplx Y = conj(FT(it, k1, mup));
                        acc1 += creal(Y * o->eb[((size_t)(k1 * nphi + k2) * nphi + j2) * npsi + j1]);
                    }
                }
                ov[(it * nphi + j2) * npsi + j1] = acc0 + 2.0 * acc1;
            }
#undef FT
}

int orc_angl2proj(const orc *o, const double *ov, double *p /* complex */)
{
    cplx *ft = malloc(sizeof(cplx) * o->ntheta * o->nmu2 * (2 * o->mmax + 1));
    angl2proj_pt(o, ov, (cplx *)p, ft);
    free(ft);
    return 0;
}
int orc_proj2angl(const orc *o, const double *p, double *ov)
{
    cplx *ft = malloc(sizeof(cplx) * o->ntheta * o->nmu2 * (2 * o->mmax + 1));
    proj2angl_pt(o, (const cplx *)p, ov, ft);
    free(ft);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* The rotated OZ step for one (q, -q) pair: module_energy_cproj_mrso.f90:   */
/* 476-661.  Fortran `cmplx(x,y)` without KIND yields default (single)       */
/* precision, so the flushed entries keep only the FP32-rounded other part.  */
static inline double to_sp(double x) { return (double)(float)x; }
/* Diagnostic switch (tests only): bit 0 keeps the FP32 rounding of the R flush,
   bit 1 keeps the FP32 rounding of the gamma flush.  Default: both, as in the reference. */
static int g_quirks = 3;
void orc_set_quirks(int q) { g_quirks = q; }
static inline double q_sp(double x, int bit) { return (g_quirks & bit) ? to_sp(x) : x; }

/* mix = 1: the multi-species routine's form (module_energy_cproj_mrso_mixture.f90:541-557,
   :664-677), which rotates -q with R(m,mup,khi) where the single-species routine uses
   R(m,mup,-khi) (module_energy_cproj_mrso.f90:517,636). */
static void oz_pair(const orc *o, const double q[3], cplx *dq_, cplx *dmq_, int q_eq_mq, int nyq_flag, int mix,
                    cplx *outq, cplx *outmq, double *R, cplx *ceff, cplx *drq, cplx *drmq, cplx *gq, cplx *gmq)
{
    const int ks = mix ? 1 : -1; /* khi of the -q rotation is ks*khi */
    const int M = o->mmax, W = 2 * M + 1, np = o->np, mrso = o->mrso;
    orc_rotation_matrix(M, q, R);
    const int sz = (M + 1) * W * W;
    for (int i = 0; i < sz; ++i) { /* :491-492 */
        if (fabs(R[2 * i]) < EPSSP) { R[2 * i] = 0.0; R[2 * i + 1] = q_sp(R[2 * i + 1], 1); }
        if (fabs(R[2 * i + 1]) < EPSSP) { R[2 * i] = q_sp(R[2 * i], 1); R[2 * i + 1] = 0.0; }
    }
#define RR(m, mup, khi) (R[2 * RIDX(m, mup, khi, M)] + I * R[2 * RIDX(m, mup, khi, M) + 1])
    /* forward rotation :505-523 (gq, gmq hold the lab-frame projections) */
    for (int i = 0; i < np; ++i) { gq[i] = dq_[i]; gmq[i] = dmq_[i]; }
    int ip = 0;
    for (int m = 0; m <= M; ++m)
        for (int khi = -m; khi <= m; ++khi)
            for (int mu2 = 0; mu2 <= m / mrso; ++mu2, ++ip) {
                cplx a = 0, b = 0;
                for (int mup = -m; mup <= m; ++mup) {
                    int jp = o->p3p[p3idx(o, m, mup, mu2)];
                    a = a + gq[jp] * RR(m, mup, khi);
                    b = b + gmq[jp] * RR(m, mup, ks * khi);
                }
                drq[ip] = a;
                drmq[ip] = b * ((m % 2 == 0) ? 1.0 : -1.0);
            }
    /* interpolated c :534-539 */
    double nq = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
    double effectiveiq = nq / o->dq + 1.0;
    int iq = (int)effectiveiq;
    double alpha = effectiveiq - iq;
    const cplx *c0 = o->c + (size_t)(iq - 1) * o->ncoef, *c1 = o->c + (size_t)iq * o->ncoef;
    for (int k = 0; k < o->ncoef; ++k) ceff[k] = alpha * c1[k] + (1.0 - alpha) * c0[k];
    /* OZ :561-606 */
    int ia = 0;
    for (ip = 0; ip < np; ++ip) {
        int m = o->p3m[ip], khi = o->p3mup[ip];
        (void)m;
        cplx a = 0, b = 0;
        for (int n = abs(khi); n <= M; ++n)
            for (int nu2 = -n / mrso; nu2 <= n / mrso; ++nu2, ++ia) {
                if (nu2 < 0) {
                    int jp = o->p3p[p3idx(o, n, khi, -nu2)];
                    a = a + ceff[ia] * drq[jp];
                    b = b + ceff[ia] * drmq[jp];
                } else {
                    int jp = o->p3p[p3idx(o, n, khi, nu2)];
                    a = a + ceff[ia] * conj(drmq[jp]);
                    b = b + ceff[ia] * conj(drq[jp]);
                }
            }
        gq[ip] = a;
        gmq[ip] = b;
    }
    /* underflow flush :618-623 */
    for (ip = 0; ip < np; ++ip) {
        cplx *v[2] = {&gq[ip], &gmq[ip]};
        for (int t = 0; t < 2; ++t) {
            double re = creal(*v[t]), im = cimag(*v[t]);
            if (fabs(re) < EPSDP && fabs(im) < EPSDP) { re = 0; im = 0; }
            if (fabs(re) < EPSDP) { re = 0.0; im = q_sp(im, 2); }
            if (fabs(im) < EPSDP) { re = q_sp(re, 2); im = 0.0; }
            *v[t] = re + I * im;
        }
    }
    /* back rotation with conj(R) :611-641 */
    ip = 0;
    for (int m = 0; m <= M; ++m)
        for (int mup = -m; mup <= m; ++mup)
            for (int mu2 = 0; mu2 <= m / mrso; ++mu2, ++ip) {
                cplx a = 0, b = 0;
                for (int khi = -m; khi <= m; ++khi) {
                    int jp = o->p3p[p3idx(o, m, khi, mu2)];
                    a = a + gq[jp] * conj(RR(m, mup, khi));
                    b = b + gmq[jp] * conj(RR(m, mup, ks * khi));
                }
                outq[ip] = a;
                outmq[ip] = b * ((m % 2 == 0) ? 1.0 : -1.0);
            }
    if (q_eq_mq && nyq_flag)
        for (ip = 0; ip < np; ++ip) outmq[ip] = conj(outmq[ip]);
#undef RR
}

/* ------------------------------------------------------------------------- */
/* The stages of energy_cproj_mrso (module_energy_cproj_mrso.f90:61-782),    */
/* shared with energy_cproj_mrso_mixture.                                    */

/* S1 projection of rho0 (xi^2 - 1) (:276-290) and S2 forward FFT, sign +1 (:306-329). */
static void project_forward(const orc *o, const double *xi, cplx *drho /* [N][np] ip fastest */)
{
    const int nx = o->nx, ny = o->ny, nz = o->nz, np = o->np, no = o->no;
    const long N = o->N;
    const double rho0 = o->rho0;
#pragma omp parallel
    {
        double *ov = malloc(sizeof(double) * no);
        cplx *ft = malloc(sizeof(cplx) * o->ntheta * o->nmu2 * (2 * o->mmax + 1));
#pragma omp for
        for (long r = 0; r < N; ++r) {
            for (int io = 0; io < no; ++io) {
                double x = xi[r * no + io];
                ov[io] = rho0 * (x * x - 1.0);
            }
            angl2proj_pt(o, ov, drho + r * np, ft);
        }
        free(ov);
        free(ft);
    }
    cplx *buf = malloc(sizeof(cplx) * N);
    for (int ip = 0; ip < np; ++ip) {
        for (long r = 0; r < N; ++r) buf[r] = drho[r * np + ip];
        fft3d(buf, nx, ny, nz, +1);
        for (long r = 0; r < N; ++r) drho[r * np + ip] = buf[r];
    }
    free(buf);
}

/* S3-S5, every (q, -q) pair once, in the reference's serial order, with oc's c table.
   mix = 0 (module_energy_cproj_mrso.f90:462-665): in place (out == in); the -q result
   replaces the q result at self-conjugate points, conjugated where a Nyquist index is set.
   mix = 1 (module_energy_cproj_mrso_mixture.f90:491-721): out += the results; at
   self-conjugate points only the q result is added. */
static int oz_sweep(const orc *oc, const cplx *in, cplx *out, int mix)
{
    const int nx = oc->nx, ny = oc->ny, nz = oc->nz, np = oc->np;
    const long N = oc->N;
    char *isok = calloc(N, 1);
    const int M = oc->mmax, W = 2 * M + 1;
    double *R = malloc(sizeof(double) * 2 * (M + 1) * W * W);
    cplx *ceff = malloc(sizeof(cplx) * oc->ncoef);
    cplx *tmp = malloc(sizeof(cplx) * 8 * np);
    cplx *drq = tmp, *drmq = tmp + np, *gq = tmp + 2 * np, *gmq = tmp + 3 * np;
    cplx *oq = tmp + 4 * np, *omq = tmp + 5 * np, *inq = tmp + 6 * np, *inmq = tmp + 7 * np;
    for (int izq = 1; izq <= nz / 2 + 1; ++izq) {
        int izmq = (izq == 1) ? 1 : nz - izq + 2;
        for (int iyq = 1; iyq <= ny; ++iyq) {
            int iymq = (iyq == 1) ? 1 : ny - iyq + 2;
            for (int ixq = 1; ixq <= nx; ++ixq) {
                int ixmq = (ixq == 1) ? 1 : nx - ixq + 2;
                long rq = ((long)(izq - 1) * ny + (iyq - 1)) * nx + (ixq - 1);
                long rmq = ((long)(izmq - 1) * ny + (iymq - 1)) * nx + (ixmq - 1);
                if (isok[rq] && isok[rmq]) continue;
                int q_eq_mq = (ixmq == ixq && iymq == iyq && izmq == izq);
                int nyq = (ixq == nx / 2 + 1 || iyq == ny / 2 + 1 || izq == nz / 2 + 1);
                double q[3] = {oc->kx[ixq - 1], oc->ky[iyq - 1], oc->kz[izq - 1]};
                for (int i = 0; i < np; ++i) { inq[i] = in[rq * np + i]; inmq[i] = in[rmq * np + i]; }
                oz_pair(oc, q, inq, inmq, q_eq_mq, mix ? 0 : nyq, mix, oq, omq, R, ceff, drq, drmq, gq, gmq);
                if (mix) {
                    for (int i = 0; i < np; ++i) out[rq * np + i] += oq[i];
                    if (!q_eq_mq)
                        for (int i = 0; i < np; ++i) out[rmq * np + i] += omq[i];
                } else {
                    for (int i = 0; i < np; ++i) out[rq * np + i] = oq[i];
                    for (int i = 0; i < np; ++i) out[rmq * np + i] = omq[i];
                }
                isok[rq] = 1;
                isok[rmq] = 1;
            }
        }
    }
    int rc = 0;
    for (long r = 0; r < N; ++r)
        if (!isok[r]) { set_err("not all gamma_p computed"); rc = -1; break; }
    free(isok); free(R); free(ceff); free(tmp);
    return rc;
}

/* S6 inverse FFT, sign -1, times 1/N (:690-719). */
static void inverse_fft(const orc *o, cplx *drho)
{
    const int nx = o->nx, ny = o->ny, nz = o->nz, np = o->np;
    const long N = o->N;
    const double cst = 1.0 / (double)(nx * ny * nz);
    cplx *buf = malloc(sizeof(cplx) * N);
    for (int ip = 0; ip < np; ++ip) {
        for (long r = 0; r < N; ++r) buf[r] = drho[r * np + ip];
        fft3d(buf, nx, ny, nz, -1);
        for (long r = 0; r < N; ++r) drho[r * np + ip] = buf[r] * cst;
    }
    free(buf);
}

/* S7 gather (:728-762): returns sum (xi^2 rho0 - rho0) v with v = prefactor w proj2angl(gamma),
   and adds 2 rho0 xi v to df. */
static double gather_excess(const orc *o, const cplx *drho, const double *xi, double prefactor, double *df)
{
    const int np = o->np, no = o->no;
    const long N = o->N;
    const double rho0 = o->rho0;
    double pff[ORC_NCHUNK];
#pragma omp parallel
    {
        double *vexc = malloc(sizeof(double) * no);
        cplx *ft = malloc(sizeof(cplx) * o->ntheta * o->nmu2 * (2 * o->mmax + 1));
#pragma omp for
        for (int ch = 0; ch < ORC_NCHUNK; ++ch) {
          double ff = 0.0;
          for (long r = N * ch / ORC_NCHUNK; r < N * (ch + 1) / ORC_NCHUNK; ++r) {
            proj2angl_pt(o, drho + r * np, vexc, ft);
            double s = 0;
            for (int io = 0; io < no; ++io) {
                double v = prefactor * o->w[io] * vexc[io];
                double x = xi[r * no + io];
                s += (x * x * rho0 - rho0) * v;
                if (df) df[r * no + io] = df[r * no + io] + 2.0 * rho0 * x * v;
            }
            ff += s;
          }
          pff[ch] = ff;
        }
        free(vexc);
        free(ft);
    }
    double ff = 0.0;
    for (int ch = 0; ch < ORC_NCHUNK; ++ch) ff += pff[ch];
    return ff;
}

/* energy_cproj_mrso: module_energy_cproj_mrso.f90:61-782. */
static int excess(orc *o, const double *xi, double *fexc, double *df)
{
    if (!o->c) { set_err("c(k) table not loaded"); return -1; }
    project_forward(o, xi, o->drho);
    if (oz_sweep(o, o->drho, o->drho, 0)) return -1;
    inverse_fft(o, o->drho);
    const double fourpisq = 4.0 * ORC_PI * ORC_PI;
    const double prefactor = -o->kT * 2.0 * fourpisq / o->mrso / o->n0;
    *fexc = gather_excess(o, o->drho, xi, prefactor, df) * 0.5 * o->dv;
    return 0;
}

/* energy_cproj_mrso_mixture: module_energy_cproj_mrso_mixture.f90:67-850.  sp[s] holds species
   s (its n0 already times its mole fraction, module_solvent.f90:221-222, its c table and
   vext); xi and df are [ns][N][no].  gamma_{s2} = sum_s OZ_{c(s2)}(drho_s), summed in the
   reference's order (s outer, s2 inner, :491-721), then gathered per s2 with the prefactor
   -kT 2 (4 pi^2) / mrso / n0(s2) x(s2) (:788-809). */
static int excess_mixture(orc *const *sp, int ns, const double *xfrac, const double *xi, double *fexc, double *df)
{
    const orc *o = sp[0];
    const long N = o->N, no = o->no, np = o->np;
    for (int s = 0; s < ns; ++s)
        if (!sp[s]->c) { set_err("c(k) table not loaded"); return -1; }
    cplx *gam = calloc((size_t)ns * N * np, sizeof(cplx));
    if (!gam) { set_err("out of memory"); return -1; }
    for (int s = 0; s < ns; ++s) project_forward(sp[s], xi + s * N * no, sp[s]->drho);
    for (int s = 0; s < ns; ++s)
        for (int s2 = 0; s2 < ns; ++s2)
            if (oz_sweep(sp[s2], sp[s]->drho, gam + s2 * N * np, 1)) { free(gam); return -1; }
    const double fourpisq = 4.0 * ORC_PI * ORC_PI;
    double ff = 0.0;
    for (int s2 = 0; s2 < ns; ++s2) {
        inverse_fft(o, gam + s2 * N * np);
        const double prefactor = -sp[s2]->kT * 2.0 * fourpisq / sp[s2]->mrso / sp[s2]->n0 * xfrac[s2];
        ff += gather_excess(sp[s2], gam + s2 * N * np, xi + s2 * N * no, prefactor, df ? df + s2 * N * no : NULL);
    }
    free(gam);
    *fexc = ff * 0.5 * o->dv;
    return 0;
}

/* module_energy_ideal_and_external.f90:14-74 */
static void ideal_and_external(const orc *o, const double *xi, double *fid, double *fext, double *df)
{
    const double kT = o->kT, dv = o->dv, rho0 = o->rho0;
    const int no = o->no;
    double pa[ORC_NCHUNK], pb[ORC_NCHUNK];
#pragma omp parallel for
    for (int ch = 0; ch < ORC_NCHUNK; ++ch) {
      double a = 0, b = 0;
      for (long r = o->N * ch / ORC_NCHUNK; r < o->N * (ch + 1) / ORC_NCHUNK; ++r)
        for (int io = 0; io < no; ++io) {
            long i = r * no + io;
            double x = xi[i], rho = x * x * rho0;
            if (rho > EPSDP) {
                a += kT * dv * o->w[io] * (rho * log(rho / rho0) - rho + rho0);
                b += dv * o->w[io] * rho * o->vext[i];
                if (df) df[i] = df[i] + o->w[io] * 2.0 * rho0 * x * (kT * log(rho / rho0) + o->vext[i]);
            } else {
                a += kT * dv * o->w[io] * rho0;
            }
        }
      pa[ch] = a;
      pb[ch] = b;
    }
    double a = 0, b = 0;
    for (int ch = 0; ch < ORC_NCHUNK; ++ch) { a += pa[ch]; b += pb[ch]; }
    *fid = a;
    *fext = b;
}

/* energy_and_gradient: module_energy_and_gradient.f90:36-240.               */
/* terms = {F_id, F_ext, F_exc, corrections}                                  */
static int bridge_cgb(const orc *o, const double *xi, double *fb, double *df);
static int bridge_fmt(const orc *o, const double *xi, double *fb, double *df);

int orc_energy_grad(orc *o, const double *xi, double *f, double *df, double *terms)
{
    if (df) memset(df, 0, sizeof(double) * o->N * o->no);
    double fid, fext, fexc, fb = 0.0;
    ideal_and_external(o, xi, &fid, &fext, df);
    if (excess(o, xi, &fexc, df)) return -1;
    if (o->cgb && bridge_cgb(o, xi, &fb, df)) return -1; /* energy_bridge :166-175, :246-275 */
    if (o->fmt && bridge_fmt(o, xi, &fb, df)) return -1;
    double ff = 0.0;
    ff = ff + fid + fext;
    ff = ff + fexc;
    ff = ff + fb;
    ff = ff + o->const_corr;
    *f = ff;
    if (terms) { terms[0] = fid; terms[1] = fext; terms[2] = fexc; terms[3] = o->const_corr; }
    return 0;
}

/* energy_and_gradient with nspec > 1 species (module_energy_and_gradient.f90:86-217 with the
   excess pointer on energy_cproj_mrso_mixture, module_init_simu.f90:67-71): the ideal and
   external terms summed over species (module_energy_ideal_and_external.f90:46-72), then the
   mixture excess.  xi, df: [ns][N][no]; the constant corrections are sp[0]'s.  The oracle
   accepts ns = 1 too (the mixture routine's own form of one species). */
int orc_mixture_energy_grad(orc *const *sp, int ns, const double *xfrac, const double *xi, double *f, double *df,
                            double *terms)
{
    if (ns < 1 || !sp || !xfrac) { set_err("bad species list"); return -1; }
    const orc *o = sp[0];
    double xs = 0.0;
    for (int s = 0; s < ns; ++s) {
        const orc *p = sp[s];
        if (!p || p->nx != o->nx || p->ny != o->ny || p->nz != o->nz || p->lx != o->lx || p->ly != o->ly ||
            p->lz != o->lz || p->mmax != o->mmax || p->mrso != o->mrso || p->kT != o->kT) {
            set_err("species differ in grid, angular order or temperature");
            return -1;
        }
        if (!(xfrac[s] > 0.0 && xfrac[s] <= 1.0)) { set_err("mole fraction outside (0, 1]"); return -1; }
        xs += xfrac[s];
    }
    if (xs != 1.0) { set_err("mole fractions do not sum to 1"); return -1; }
    const long n = o->N * o->no;
    if (df) memset(df, 0, sizeof(double) * n * ns);
    double fid = 0.0, fext = 0.0, fexc;
    for (int s = 0; s < ns; ++s) {
        double a, b;
        ideal_and_external(sp[s], xi + s * n, &a, &b, df ? df + s * n : NULL);
        fid += a;
        fext += b;
    }
    if (excess_mixture(sp, ns, xfrac, xi, &fexc, df)) return -1;
    double ff = 0.0;
    ff = ff + fid + fext;
    ff = ff + fexc;
    ff = ff + 0.0; /* bridge "no" */
    ff = ff + o->const_corr;
    *f = ff;
    if (terms) { terms[0] = fid; terms[1] = fext; terms[2] = fexc; terms[3] = o->const_corr; }
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Coarse-grained bridge, bridge = "cgb":                                     */
/* module_coarse_grained_gageat_bridge.f90:50-482 (one species).             */

/* fill_kernel (:123-210): the normalised Gaussian of width sigma on the periodic grid,
   cut where it falls below 1e-10, forward transformed (r2c, sign -1) and scaled by
   V / real(N) -- `real(nx*ny*nz)` is single precision. */
static void cgb_kernel_k(const orc *o, double sigma, cplx *kk)
{
    const double pi = acos(-1.0);
    const double sp = sigma * sqrt(2.0 * pi);
    const double gp = 1.0 / (sp * sp * sp);
    const double oo = 1.0 / (2.0 * sigma * sigma);
    const double cut = -1.0 / oo * log(1.0e-10 / gp);
    const int nx = o->nx, ny = o->ny, nz = o->nz;
    for (int iz = 0; iz < nz; ++iz)
        for (int iy = 0; iy < ny; ++iy)
            for (int ix = 0; ix < nx; ++ix) {
                const double xp = o->dx * (ix < nx - ix ? ix : nx - ix);
                const double yp = o->dy * (iy < ny - iy ? iy : ny - iy);
                const double zp = o->dz * (iz < nz - iz ? iz : nz - iz);
                const double d2 = xp * xp + yp * yp + zp * zp;
                kk[((long)iz * ny + iy) * nx + ix] = d2 < cut ? gp * exp(-d2 * oo) : 0.0;
            }
    fft3d(kk, nx, ny, nz, -1);
    const double nf = (double)(float)(nx * ny * nz), vol = o->lx * o->ly * o->lz;
    for (long r = 0; r < o->N; ++r) kk[r] = kk[r] / nf * vol;
}

/* out = c2r(r2c(in) * kernel_k) / real(N) (:424-451), as a complex FFT of real data. */
static void cgb_convolve(const orc *o, const cplx *kk, const double *in, double *out, cplx *buf)
{
    for (long r = 0; r < o->N; ++r) buf[r] = in[r];
    fft3d(buf, o->nx, o->ny, o->nz, -1);
    for (long r = 0; r < o->N; ++r) buf[r] *= kk[r];
    fft3d(buf, o->nx, o->ny, o->nz, +1);
    const double nf = (double)(float)(o->nx * o->ny * o->nz);
    for (long r = 0; r < o->N; ++r) out[r] = creal(buf[r]) / nf;
}

/* coarse_grained_bridge (:216-421); df (may be NULL) accumulates 2 xi rho0 dfb w (:455-482). */
static int bridge_cgb(const orc *o, const double *xi, double *fb_out, double *df)
{
    const long N = o->N;
    const int no = o->no;
    const double kT = o->kT, n0 = o->n0, rho0 = o->rho0;
    const double vvox = o->dx * o->dy * o->dz, facteur = kT * vvox;
    const double A3 = 1.0 - o->cgb_c00 / 2.0, B6 = o->cgb_B6;
    cplx *kk = malloc(sizeof(cplx) * N), *buf = malloc(sizeof(cplx) * N);
    double *dens = calloc(N, sizeof(double)), *dcg = calloc(N, sizeof(double));
    double *t = calloc(N, sizeof(double)), *dfb = calloc(N, sizeof(double));
    if (!kk || !buf || !dens || !dcg || !t || !dfb) {
        free(kk); free(buf); free(dens); free(dcg); free(t); free(dfb);
        set_err("out of memory");
        return -1;
    }
    cgb_kernel_k(o, o->cgb_sigma, kk);
    /* integrate_over_orientations(xi**2 * rho0) / n0 (module_grid.f90:354-380) */
    for (long r = 0; r < N; ++r) {
        double a = 0.0;
        for (int io = 0; io < no; ++io) {
            const double x = xi[r * no + io];
            a += x * x * rho0 * o->w[io];
        }
        dens[r] = a / n0;
    }
    cgb_convolve(o, kk, dens, dcg, buf);
    double fb = 0.0;
    if (o->cgb == 1) { /* 'sla' (:274-347) */
        for (long r = 0; r < N; ++r) {
            const double ncg = dcg[r], dn = ncg - 1.0;
            double phib, d;
            if (ncg < 1.0) {
                phib = A3 * (dn * dn * dn) + B6 * (ncg * ncg) * ((dn * dn) * (dn * dn));
                d = kT * A3 * 3.0 * (dn * dn) + kT * B6 * (2.0 * ncg * ((dn * dn) * (dn * dn)) + 4.0 * (ncg * ncg) * (dn * dn * dn));
            } else {
                phib = A3 * (dn * dn * dn);
                d = kT * A3 * 3.0 * (dn * dn);
            }
            fb = fb + facteur * n0 * phib;
            t[r] = d;
        }
        if (df) cgb_convolve(o, kk, t, dfb, buf);
    } else { /* 'wda' (:349-419) */
        if (df) {
            for (long r = 0; r < N; ++r) {
                const double ncg = dcg[r], dn = ncg - 1.0;
                t[r] = ncg < 1.0 ? A3 * 2.0 * dn + B6 * (2.0 * ncg * (dn * dn * dn) + 3.0 * (ncg * ncg) * (dn * dn))
                                 : A3 * 2.0 * dn;
            }
            cgb_convolve(o, kk, t, dfb, buf);
        }
        for (long r = 0; r < N; ++r) {
            const double ncg = dcg[r], dN = dens[r] - 1.0, dn = ncg - 1.0;
            const double phib = ncg < 1.0 ? A3 * (dn * dn) + B6 * (ncg * ncg) * (dn * dn * dn) : A3 * (dn * dn);
            fb = fb + kT * vvox * n0 * dN * phib;
            if (df) t[r] = kT * (dN * dfb[r] + phib);
        }
        if (df) memcpy(dfb, t, sizeof(double) * N);
    }
    if (df)
        for (long r = 0; r < N; ++r)
            for (int io = 0; io < no; ++io) df[r * no + io] = df[r * no + io] + 2.0 * xi[r * no + io] * rho0 * dfb[r] * o->w[io];
    free(kk); free(buf); free(dens); free(dcg); free(t); free(dfb);
    *fb_out = fb;
    return 0;
}

/* version 0 removes the bridge (bridge = "no"), 1 'sla', 2 'wda' (cgb_version, :72). */
int orc_set_bridge_cgb(orc *o, int version, double B6, double sigma, double c00)
{
    if (version < 0 || version > 2 || !(sigma > 0.0)) { set_err("bad cgb parameters"); return -1; }
    o->cgb = version;
    o->cgb_B6 = B6;
    o->cgb_sigma = sigma;
    o->cgb_c00 = c00;
    return 0;
}

/* energy_bridge(fb, df) alone: fb and df += the bridge's gradient (df may be NULL). */
int orc_bridge_energy(orc *o, const double *xi, double *fb, double *df)
{
    *fb = 0.0;
    if (o->cgb) return bridge_cgb(o, xi, fb, df);
    if (o->fmt) return bridge_fmt(o, xi, fb, df);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Hard-sphere bridge, bridge = "hard_sphere" (one species): module_fmt.f90:5-317 with the   */
/* Kierlik-Rosinberg weights of module_hardspheres.f90:40-73, the bulk parameters of        */
/* :83-189 and the hard-sphere c(k) of cs_of_k_hard_sphere.f90:3-166.                      */

/* w_alpha(k), module_hardspheres.f90:56-70 */
static void hs_weights(double R, double k, double w[4])
{
    const double fourpi = 4.0 * ORC_PI;
    if (fabs(k) > EPSDP) {
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

/* functional 1 PY, 2 CS; 0 removes the term.  dq: the c(k) file's step, as module_grid's dq
   after energy_cproj_mrso (module_energy_cproj_mrso.f90:369). */
int orc_set_bridge_fmt(orc *o, int functional, double R)
{
    free(o->hs_cs);
    o->hs_cs = NULL;
    o->fmt = 0;
    if (functional == 0) return 0;
    if (functional < 0 || functional > 2 || !(R > 0.0)) { set_err("bad hard-sphere parameters"); return -1; }
    if (!o->c) { set_err("c(k) table not loaded"); return -1; }
    const double pi = ORC_PI, kT = o->kT, n0b = o->n0;
    /* packing fraction (:19-28, fourthird = 4./3. in single precision) and its limit (:113-120) */
    const double pf = (double)(4.0f / 3.0f) * pi * n0b * (R * R * R);
    if (pf >= 0.74) { set_err("hard-sphere packing fraction above 0.74"); return -1; }
    /* excess chemical potential and bulk grand potential (:136-187) */
    const double n0 = n0b, n1 = n0 * R, n2 = n0 * 4 * pi * (R * R), n3 = n0 * 4 * pi * (R * R * R) / 3;
    double dphi[4];
    if (functional == 1) {
        dphi[0] = -log(1 - n3);
        dphi[1] = n2 / (1 - n3);
        dphi[2] = n1 / (1 - n3) + (n2 * n2) / (8 * pi * ((1 - n3) * (1 - n3)));
        dphi[3] = n0 / (1 - n3) + n1 * n2 / ((1 - n3) * (1 - n3)) + (n2 * n2 * n2) / (12 * pi * ((1 - n3) * (1 - n3) * (1 - n3)));
    } else {
        const double m1 = n3 - 1;
        dphi[0] = -log(1 - n3);
        dphi[1] = n2 / (1 - n3);
        dphi[2] = (n3 * ((n2 * n2) - 12 * n1 * m1 * n3 * pi) + (n2 * n2) * (m1 * m1) * log(1 - n3)) / (12 * pi * (m1 * m1) * (n3 * n3));
        dphi[3] = (n3 * ((n2 * n2 * n2) * (2 - 5 * n3 + (n3 * n3)) + 36 * n1 * n2 * m1 * (n3 * n3) * pi - 36 * n0 * (m1 * m1) * (n3 * n3) * pi) -
                   2 * (n2 * n2 * n2) * (m1 * m1 * m1) * log(1 - n3)) /
                  (36 * pi * (m1 * m1 * m1) * (n3 * n3 * n3));
    }
    const double dndrho[4] = {1, R, 4 * pi * (R * R), 4 * pi * (R * R * R) / 3.0};
    double acc = 0.0;
    for (int a = 0; a < 4; ++a) acc += dphi[a] * dndrho[a];
    const double mu = kT * acc;
    double fexc0;
    if (functional == 1)
        fexc0 = kT * (-n0 * log(1 - n3) + n1 * n2 / (1 - n3) + (n2 * n2 * n2) / (24 * pi * ((1 - n3) * (1 - n3))));
    else
        fexc0 = kT * (((1.0 / (36 * pi)) * (n2 * n2 * n2) / (n3 * n3) - n0) * log(1 - n3) + n1 * n2 / (1 - n3) +
                      (1.0 / (36 * pi)) * (n2 * n2 * n2) / (((1 - n3) * (1 - n3)) * n3));
    fexc0 = (fexc0 - mu * n0b) * (o->lx * o->ly * o->lz);
    /* the hard-sphere c(k) (cs_of_k_hard_sphere.f90:56-157) */
    const double kxm = o->kx[o->nx / 2], kym = o->ky[o->ny / 2], kzm = o->kz[o->nz / 2];
    const int nbk = (int)(sqrt(kxm * kxm + kym * kym + kzm * kzm) / o->dq) + 1;
    double *cs = malloc(sizeof(double) * nbk);
    if (!cs) { set_err("out of memory"); return -1; }
    double b0 = 0, b1 = 0, b2 = 0, b3 = 0; /* the bulk weighted densities, set at k = 0 */
    for (int i = 0; i < nbk; ++i) {
        const double k = i * o->dq;
        double w[4];
        if (fabs(k) <= EPSDP) {
            w[0] = 1.0; w[1] = R; w[2] = 4.0 * pi * (R * R); w[3] = 4.0 * pi / 3.0 * (R * R * R);
            b0 = n0b * w[0]; b1 = n0b * w[1]; b2 = n0b * w[2]; b3 = n0b * w[3];
        } else {
            const double kR = k * R, sk = sin(kR), ck = cos(kR);
            w[0] = ck + kR * sk / 2.0;
            w[1] = (sk + kR * ck) / (2.0 * k);
            w[2] = (4.0 * pi * R * sk) / k;
            w[3] = 4.0 * pi * (sk - kR * ck) / (k * k * k);
        }
        if (fabs(b3 - 1) <= EPSDP) { free(cs); set_err("n3 = 1 in the hard-sphere c(k)"); return -1; }
        double d[4][4] = {{0}};
        const double u = 1.0 - b3;
        if (functional == 1) {
            d[0][3] = 1.0 / u;
            d[1][2] = 1.0 / u;
            d[1][3] = b2 / (u * u);
            d[2][1] = d[1][2];
            d[2][2] = b2 / (4 * pi * (u * u));
            d[2][3] = b1 / (u * u) + (b2 * b2) / (4 * pi * (u * u * u));
            d[3][0] = d[0][3];
            d[3][1] = d[1][3];
            d[3][2] = d[2][3];
            d[3][3] = (2.0 * b1 * b2) / (u * u * u) + b0 / (u * u) + (b2 * b2 * b2) / (4.0 * pi * ((u * u) * (u * u)));
        } else {
            const double m1 = -1.0 + b3;
            d[0][3] = 1.0 / (1 - b3);
            d[1][2] = 1.0 / (1.0 - b3);
            d[1][3] = b2 / ((1.0 - b3) * (1.0 - b3));
            d[2][1] = d[1][2];
            d[2][2] = b2 / (6.0 * ((1.0 - b3) * (1.0 - b3)) * b3 * pi) + (b2 * log(1.0 - b3)) / (6.0 * (b3 * b3) * pi);
            d[2][3] = (b3 * ((b2 * b2) * (2.0 - 5.0 * b3 + (b3 * b3)) + 12.0 * b1 * m1 * (b3 * b3) * pi) -
                       2.0 * (b2 * b2) * (m1 * m1 * m1) * log(1 - b3)) /
                      (12.0 * (m1 * m1 * m1) * (b3 * b3 * b3) * pi);
            d[3][0] = d[0][3];
            d[3][1] = d[1][3];
            d[3][2] = d[2][3];
            d[3][3] = (b3 * ((b2 * b2 * b2) * (6.0 - 21.0 * b3 + 26.0 * (b3 * b3) - 5.0 * (b3 * b3 * b3)) -
                             72.0 * b1 * b2 * m1 * (b3 * b3 * b3) * pi + 36.0 * b0 * (m1 * m1) * (b3 * b3 * b3) * pi) +
                       6.0 * (b2 * b2 * b2) * ((m1 * m1) * (m1 * m1)) * log(1.0 - b3)) /
                      (36.0 * ((m1 * m1) * (m1 * m1)) * ((b3 * b3) * (b3 * b3)) * pi);
        }
        double sum = 0.0;
        for (int a = 0; a < 4; ++a)
            for (int b = 0; b < 4; ++b) sum += d[a][b] * w[a] * w[b];
        cs[i] = -sum;
    }
    o->fmt = functional;
    o->hs_R = R;
    o->hs_mu = mu;
    o->hs_fexc0 = fexc0;
    o->hs_nbk = nbk;
    o->hs_cs = cs;
    return 0;
}

int orc_fmt_params(const orc *o, double *out /* R, mu, Fexc0, nb_k */)
{
    out[0] = o->hs_R; out[1] = o->hs_mu; out[2] = o->hs_fexc0; out[3] = o->hs_nbk;
    return o->fmt ? 0 : -1;
}

/* energy_bridge_fmt (module_fmt.f90:5-317) for one species (mole fraction 1).  Real-to-complex
   transforms run as complex FFTs of real data; the multipliers depend on |k| only. */
static int bridge_fmt(const orc *o, const double *xi, double *fb_out, double *df)
{
    const long N = o->N;
    const int no = o->no, nx = o->nx, ny = o->ny, nz = o->nz;
    const double kT = o->kT, dv = o->dv, rho0 = o->rho0, pi = ORC_PI, R = o->hs_R, mu = o->hs_mu;
    /* empty box (:46-49) */
    int empty = 1;
    for (long i = 0; i < N * no && empty; ++i)
        if (fabs(xi[i]) > EPSDP) empty = 0;
    if (empty) { *fb_out = -o->hs_fexc0; return 0; }
    cplx *rk = malloc(sizeof(cplx) * N), *wd = malloc(sizeof(cplx) * 4 * N), *gk = malloc(sizeof(cplx) * N);
    double *rho = calloc(N, sizeof(double)), *kn = malloc(sizeof(double) * N);
    if (!rk || !wd || !gk || !rho || !kn) {
        free(rk); free(wd); free(gk); free(rho); free(kn);
        set_err("out of memory");
        return -1;
    }
    for (int iz = 0; iz < nz; ++iz)
        for (int iy = 0; iy < ny; ++iy)
            for (int ix = 0; ix < nx; ++ix) {
                const double kx = o->kx[ix], ky = o->ky[iy], kz = o->kz[iz];
                kn[((long)iz * ny + iy) * nx + ix] = sqrt(kx * kx + ky * ky + kz * kz);
            }
    /* rho(r) = sum_io xi^2 w (:51-63) and the molecule count (:66-68) */
    double srho = 0.0;
    for (long r = 0; r < N; ++r) {
        double a = 0.0;
        for (int io = 0; io < no; ++io) a = a + xi[r * no + io] * xi[r * no + io] * o->w[io];
        rho[r] = a;
        srho += a;
    }
    const double nmol = srho * dv * rho0 * 1.0;
    /* weighted densities (:84-91) */
    for (long r = 0; r < N; ++r) rk[r] = rho[r];
    fft3d(rk, nx, ny, nz, -1);
    for (int a = 0; a < 4; ++a) {
        cplx *p = wd + a * N;
        for (long r = 0; r < N; ++r) {
            double w[4];
            hs_weights(R, kn[r], w);
            /* cmplx(w_k, 0) without KIND is single precision (:92) */
            p[r] = rk[r] * rho0 * 1.0 * (double)(float)w[a];
        }
        fft3d(p, nx, ny, nz, +1);
        for (long r = 0; r < N; ++r) p[r] = creal(p[r]) / (double)(nx * ny * nz);
    }
#define WD(a, r) creal(wd[(a) * N + (r)])
    int rc = 0;
    double s1 = 0, s2 = 0, s3 = 0;
    for (long r = 0; r < N; ++r) {
        const double w0 = WD(0, r), w1 = WD(1, r), w2 = WD(2, r), w3 = WD(3, r);
        if (w3 >= 1) { rc = -1; set_err("1 - w3 <= 0 in the hard-sphere bridge"); break; }
        if (o->fmt == 1) {
            s1 += w0 * log(1 - w3);
            s2 += w1 * w2 / (1 - w3);
            s3 += (w2 * w2 * w2) / ((1 - w3) * (1 - w3));
        } else {
            if (w3 <= EPSDP) { rc = -1; set_err("w3 <= 0 in the hard-sphere bridge"); break; }
            s1 += w1 * w2 / (1 - w3);
            s2 += ((1.0 / (36.0 * pi)) * (w2 * w2 * w2) / (w3 * w3) - w0) * log(1 - w3);
            s3 += (1.0 / (36.0 * pi)) * (w2 * w2 * w2) / (w3 * ((1 - w3) * (1 - w3)));
        }
    }
    double ffmt = 0.0;
    if (!rc) {
        ffmt = o->fmt == 1 ? -s1 + s2 + s3 / (24 * pi) : s1 + s2 + s3;
        ffmt = ffmt * kT * dv - mu * nmol - o->hs_fexc0 * 1.0;
    }
    /* gradient (:128-219): dPhi/dw_alpha, transformed, weighted, summed, back */
    if (!rc && df) {
        for (long r = 0; r < N && !rc; ++r) {
            const double w0 = WD(0, r), w1 = WD(1, r), w2 = WD(2, r), w3 = WD(3, r);
            /* :131, :138-139 */
            if ((1 - w3) <= EPSDP || (o->fmt == 2 && fabs(w3) <= EPSDP)) { rc = -1; set_err("1 - w3 or w3 at 0 in the hard-sphere bridge"); break; }
            double d[4];
            if (o->fmt == 1) {
                d[0] = -log(1 - w3);
                d[1] = w2 / (1 - w3);
                d[2] = w1 / (1 - w3) + (1.0 / (8.0 * pi)) * (d[1] * d[1]);
                d[3] = (w0 + w1 * d[1]) / (1 - w3) + (1.0 / (12.0 * pi)) * (d[1] * d[1] * d[1]);
            } else {
                const double q23 = w2 / w3;
                d[0] = -log((1 - w3));
                d[1] = w2 / (1 - w3);
                d[2] = -(1.0 / (12.0 * pi)) * (q23 * q23) * d[0] + w1 / (1 - w3) + (1.0 / (12.0 * pi)) * (d[1] * d[1]) / w3;
                d[3] = (1.0 / (18.0 * pi)) * d[0] * (q23 * q23 * q23) - ((1.0 / (36.0 * pi)) * (w2 * w2 * w2) / (w3 * w3) - w0) / (1 - w3) +
                       w1 * d[1] / (1 - w3) +
                       (1.0 / (36.0 * pi)) * (w2 * w2 * w2) / (w3 * w3) * (3.0 * w3 - 1.0) / ((1 - w3) * (1 - w3) * (1 - w3));
            }
            for (int a = 0; a < 4; ++a) wd[a * N + r] = d[a];
        }
        if (rc) goto out;
        for (int a = 0; a < 4; ++a) fft3d(wd + a * N, nx, ny, nz, -1);
        for (long r = 0; r < N; ++r) {
            double w[4];
            hs_weights(R, kn[r], w);
            gk[r] = wd[r] * w[0] + wd[N + r] * w[1] + wd[2 * N + r] * w[2] + wd[3 * N + r] * w[3];
        }
        fft3d(gk, nx, ny, nz, +1);
        for (long r = 0; r < N; ++r) {
            const double dfex = creal(gk[r]) / (double)(nx * ny * nz);
            for (int io = 0; io < no; ++io) {
                const double psi = xi[r * no + io];
                df[r * no + io] = df[r * no + io] + 2 * psi * rho0 * (kT * dfex - mu) * o->w[io];
            }
        }
    }
#undef WD
    /* minus the hard-sphere c(k)'s quadratic part (:223-282) */
    if (!rc) {
        const double shift = ((2.0 * pi) * (4.0 * pi)) / (double)o->mrso; /* twopi*fourpi/mrso */
        for (long r = 0; r < N; ++r) rk[r] = rho[r] - shift;
        fft3d(rk, nx, ny, nz, -1);
        for (long r = 0; r < N; ++r) {
            int ki = (int)(kn[r] / o->dq) + 1;
            if (ki > o->hs_nbk) ki = o->hs_nbk;
            rk[r] = rk[r] * o->hs_cs[ki - 1];
        }
        fft3d(rk, nx, ny, nz, +1);
        const double fact = dv * rho0;
        double fint = 0.0;
        for (int ix = 0; ix < nx; ++ix)
            for (int iy = 0; iy < ny; ++iy)
                for (int iz = 0; iz < nz; ++iz) {
                    const long r = ((long)iz * ny + iy) * nx + ix;
                    const double gam = creal(rk[r]) / (double)(nx * ny * nz);
                    const double vint = -kT * rho0 * gam;
                    for (int io = 0; io < no; ++io) {
                        const double psi = xi[r * no + io];
                        fint = fint + o->w[io] * fact * 0.5 * (psi * psi - 1.0) * vint;
                        if (df) df[r * no + io] = df[r * no + io] - 2.0 * psi * o->w[io] * fact * vint / dv;
                    }
                }
        ffmt = ffmt - fint;
    }
out:
    free(rk); free(wd); free(gk); free(rho); free(kn);
    *fb_out = ffmt;
    return rc;
}

/* Charged-solute corrections: module_energy_and_gradient.f90:281-344.        */
double orc_charge_corrections(double qnet, double L, double eps_r, double quad_trace, double n0)
{
    if (fabs(qnet) <= 1e-7) return 0.0;
    double pbc = -1971.01 * qnet * qnet / L * (1 - 1.0 / eps_r);
    double psch = 0.0 - quad_trace * n0 * 2909.857 * qnet;
    return pbc + psch;
}

/* ------------------------------------------------------------------------- */
/* External potential: Lennard-Jones (module_lennardjones.f90:9-226),        */
/* charges (module_solute.f90:193-236, module_fastpoissonsolver.f90:121-288, */
/* module_solvent.f90:367-438), sum + clip (module_vext.f90:600-669).         */
static const double QFACT = 1.602176565e-19 * 1.602176565e-19 * 1.0e-3 * 6.02214129e23 /
                            (4.0 * ORC_PI * 8.854187817e-12 * 1.0e-10); /* module_constants.f90:25 */
double orc_qfact(void) { return QFACT; }

int orc_vext(orc *o, int nsol, const double *sq, const double *ssig, const double *seps, const double *sxyz,
             int nsv, const double *vq, const double *vsig, const double *veps, const double *vxyz, double rvdw,
             double *lj_corr_out)
{
    const int nx = o->nx, ny = o->ny, nz = o->nz, no = o->no;
    const long N = o->N;
    const double lx = o->lx, ly = o->ly, lz = o->lz;
    double *vext = o->vext;
    memset(vext, 0, sizeof(double) * N * no);
    /* --- electrostatics first (stored apart, added in vext_total_sum) --- */
    double *vextq = NULL;
    int charged = 0;
    for (int s = 0; s < nsol; ++s) if (fabs(sq[s]) > EPSDP) charged = 1;
    if (charged) {
        vextq = calloc((size_t)N * no, sizeof(double));
        double *rhoq = calloc(N, sizeof(double));
        const double dxs[3] = {lx / nx, ly / ny, lz / nz};
        const int n3[3] = {nx, ny, nz};
        const double len[3] = {lx, ly, lz};
        for (int s = 0; s < nsol; ++s) {
            if (!(fabs(sq[s]) > EPSDP)) continue;
            double rr[3], wp[3], wm[3];
            int mi[3], pi[3];
            for (int d = 0; d < 3; ++d) {
                double x = sxyz[3 * s + d];
                rr[d] = fabs(x / dxs[d] - floor(x / dxs[d])); /* distToFloorNode */
                double md = fmod(x, len[d]);
                if (md < 0) md += len[d];
                mi[d] = (int)floor(md / dxs[d]); /* floorNode - 1 */
                pi[d] = (mi[d] + 1) % n3[d];      /* ceilingNode - 1 */
                wp[d] = rr[d];
                wm[d] = 1.0 - rr[d];
            }
            double qs = sq[s];
#define RQ(a, b, c) rhoq[((long)(c) * ny + (b)) * nx + (a)]
            RQ(mi[0], mi[1], mi[2]) += qs * wm[0] * wm[1] * wm[2];
            RQ(pi[0], mi[1], mi[2]) += qs * wp[0] * wm[1] * wm[2];
            RQ(mi[0], pi[1], mi[2]) += qs * wm[0] * wp[1] * wm[2];
            RQ(mi[0], mi[1], pi[2]) += qs * wm[0] * wm[1] * wp[2];
            RQ(pi[0], pi[1], mi[2]) += qs * wp[0] * wp[1] * wm[2];
            RQ(pi[0], mi[1], pi[2]) += qs * wp[0] * wm[1] * wp[2];
            RQ(mi[0], pi[1], pi[2]) += qs * wm[0] * wp[1] * wp[2];
            RQ(pi[0], pi[1], pi[2]) += qs * wp[0] * wp[1] * wp[2];
#undef RQ
        }
        double volumelem = (lx / nx) * (ly / ny) * (lz / nz);
        int allzero = 1;
        for (long r = 0; r < N; ++r) { rhoq[r] /= volumelem; if (fabs(rhoq[r]) > EPSDP) allzero = 0; }
        if (!allzero) {
            /* r2c (sign -1) of the density; V(k) = 4 pi rho(k)/k^2 on the half spectrum */
            cplx *rk = malloc(sizeof(cplx) * N);
            for (long r = 0; r < N; ++r) rk[r] = rhoq[r];
            fft3d(rk, nx, ny, nz, -1);
            const double twopi = 2.0 * ORC_PI, fourpi = 2.0 * twopi;
            int nxh = nx / 2 + 1;
            cplx *vk = calloc((size_t)nxh * ny * nz, sizeof(cplx));
            for (int k = 0; k < nz; ++k)
                for (int j = 0; j < ny; ++j)
                    for (int i = 0; i < nxh; ++i) {
                        int m1 = (i + 1 <= nx / 2) ? i : i - nx;
                        int m2 = (j + 1 <= ny / 2) ? j : j - ny;
                        int m3 = (k + 1 <= nz / 2) ? k : k - nz;
                        double a = twopi * m1 / lx, b = twopi * m2 / ly, c = twopi * m3 / lz;
                        double k2 = a * a + b * b + c * c;
                        cplx v = 0;
                        if (fabs(k2) > EPSDP) v = rk[((long)k * ny + j) * nx + i] * fourpi / k2;
                        vk[((long)k * ny + j) * nxh + i] = v;
                    }
            free(rk);
            /* per orientation: c2r( V(k) conj(sigma_k(io)) ) * qfact / N */
            const double smootherradius = 0.5;
            cplx *full = malloc(sizeof(cplx) * N);
            cplx *half = malloc(sizeof(cplx) * (size_t)nxh * ny * nz);
            for (int io = 0; io < no; ++io) {
                const double *R = o->rotm + 9 * io;
                for (int k = 0; k < nz; ++k)
                    for (int j = 0; j < ny; ++j)
                        for (int i = 0; i < nxh; ++i) {
                            double kv[3] = {o->kx[i], o->ky[j], o->kz[k]};
                            double sm = exp(-smootherradius * smootherradius * (kv[0] * kv[0] + kv[1] * kv[1] + kv[2] * kv[2]) / 2.0);
                            cplx sig = 0;
                            for (int n = 0; n < nsv; ++n) {
                                if (!(fabs(vq[n]) > EPSDP)) continue;
                                const double *sr = vxyz + 3 * n;
                                double r0 = R[0] * sr[0] + R[1] * sr[1] + R[2] * sr[2];
                                double r1 = R[3] * sr[0] + R[4] * sr[1] + R[5] * sr[2];
                                double r2 = R[6] * sr[0] + R[7] * sr[1] + R[8] * sr[2];
                                double kr = kv[0] * r0 + kv[1] * r1 + kv[2] * r2;
                                sig = sig + vq[n] * (cos(-kr) + I * sin(-kr)) * sm;
                            }
                            half[((long)k * ny + j) * nxh + i] = vk[((long)k * ny + j) * nxh + i] * conj(sig);
                        }
                /* Hermitian completion of the half spectrum, then c2c(+1), real part */
                for (int k = 0; k < nz; ++k)
                    for (int j = 0; j < ny; ++j)
                        for (int i = 0; i < nx; ++i) {
                            cplx v;
                            if (i < nxh) v = half[((long)k * ny + j) * nxh + i];
                            else {
                                int ii = nx - i, jj = (ny - j) % ny, kk = (nz - k) % nz;
                                v = conj(half[((long)kk * ny + jj) * nxh + ii]);
                            }
                            full[((long)k * ny + j) * nx + i] = v;
                        }
                fft3d(full, nx, ny, nz, +1);
                for (long r = 0; r < N; ++r) vextq[r * no + io] = QFACT * creal(full[r]) / (double)N;
            }
            free(full);
            free(half);
            free(vk);
        }
        free(rhoq);
    }
    /* --- Lennard-Jones (module_lennardjones.f90:9-226) --- */
    double cutoff = rvdw, cutoffsq = cutoff * cutoff;
    if (cutoff > lx * 0.5 || cutoff > ly * 0.5 || cutoff > lz * 0.5) { set_err("LJ cut-off larger than half the box"); free(vextq); return -1; }
    const double gdx = o->dx, gdy = o->dy, gdz = o->dz;
    int xts = (int)floor(2 * cutoff / gdx) + 1, yts = (int)floor(2 * cutoff / gdy) + 1, zts = (int)floor(2 * cutoff / gdz) + 1;
    int only_origin = 1;
    for (int ss = 0; ss < nsv; ++ss)
        if (veps[ss] != 0.0 && (vxyz[3 * ss] != 0.0 || vxyz[3 * ss + 1] != 0.0 || vxyz[3 * ss + 2] != 0.0)) only_origin = 0;
    double ljcorr = 0.0;
    int *tab = malloc(sizeof(int) * (nx + ny + nz + 6));
    for (int u = 0; u < nsol; ++u) {
        if (seps[u] <= EPSDP) continue;
        const double *ru = sxyz + 3 * u;
        int mn[3], mx[3];
        const double L3[3] = {lx, ly, lz}, D3[3] = {gdx, gdy, gdz};
        for (int d = 0; d < 3; ++d) {
            mn[d] = (int)floor(fmod(ru[d] - cutoff + L3[d], L3[d]) / D3[d]) + 1;
            mx[d] = (int)floor(fmod(ru[d] + cutoff, L3[d]) / D3[d]) + 1;
        }
        const int nn[3] = {nx, ny, nz};
        for (int d = 0; d < 3; ++d)
            if (mn[d] < 1 || mx[d] > nn[d]) { set_err("LJ box bound check failed"); free(tab); free(vextq); return -1; }
        /* realised index tables (Fortran reallocates on assignment); the loops below */
        /* run over the first xtabsize entries of them, as the reference does.       */
        int *xt = tab, *yt = tab + nx + 2, *ztab = tab + nx + ny + 4;
        int xlen = 0, ylen = 0, zlen = 0;
        int *tabs[3] = {xt, yt, ztab};
        int *lens[3] = {&xlen, &ylen, &zlen};
        for (int d = 0; d < 3; ++d) {
            int *t = tabs[d], n = 0;
            if (mn[d] < mx[d]) for (int i = mn[d]; i <= mx[d]; ++i) t[n++] = i;
            else { for (int i = 1; i <= mx[d]; ++i) t[n++] = i; for (int i = mn[d]; i <= nn[d]; ++i) t[n++] = i; }
            *lens[d] = n;
        }
        int xuse = xts < xlen ? xts : xlen, yuse = yts < ylen ? yts : ylen, zuse = zts < zlen ? zts : zlen;
        for (int ss = 0; ss < nsv; ++ss) {
            if (veps[ss] <= EPSDP) continue;
            double epsuv = sqrt(seps[u] * veps[ss]);
            double siguv6 = ipow((ssig[u] + vsig[ss]) * 0.5, 6);
            ljcorr = ljcorr - (16.0 * 3.14159 / 3.0) * epsuv * siguv6 * o->n0 / ipow(cutoff, 3);
            /* Serial on purpose: when the cut-off cube is as wide as the box the z table holds
               one node twice, and the reference's OpenMP loop over it races on that node. */
            for (int iz_ = 0; iz_ < zuse; ++iz_) {
                int iz = ztab[iz_] - 1;
                double zg = (double)iz * gdz;
                for (int iy_ = 0; iy_ < yuse; ++iy_) {
                    int iy = yt[iy_] - 1;
                    double yg = (double)iy * gdy;
                    for (int ix_ = 0; ix_ < xuse; ++ix_) {
                        int ix = xt[ix_] - 1;
                        double xg = (double)ix * gdx;
                        double *v = vext + (((long)iz * ny + iy) * nx + ix) * no;
                        for (int io = 0; io < no; ++io) {
                            double xs, ys, zs;
                            if (only_origin) {
                                int any = 0;
                                for (int k = 0; k < no; ++k) if (v[k] > 1.e5) any = 1;
                                if (any) break;
                                xs = xg; ys = yg; zs = zg;
                            } else {
                                if (v[io] > 1.e5) continue;
                                const double *R = o->rotm + 9 * io, *sr = vxyz + 3 * ss;
                                xs = xg + (R[0] * sr[0] + R[1] * sr[1] + R[2] * sr[2]);
                                ys = yg + (R[3] * sr[0] + R[4] * sr[1] + R[5] * sr[2]);
                                zs = zg + (R[6] * sr[0] + R[7] * sr[1] + R[8] * sr[2]);
                            }
                            double ddx = fabs(xs - ru[0]); while (ddx > lx * 0.5) ddx = fabs(ddx - lx);
                            double ddy = fabs(ys - ru[1]); while (ddy > ly * 0.5) ddy = fabs(ddy - ly);
                            double ddz = fabs(zs - ru[2]); while (ddz > lz * 0.5) ddz = fabs(ddz - lz);
                            double rsq = ddx * ddx + ddy * ddy + ddz * ddz, vlj;
                            if (rsq <= EPSDP) vlj = 1.79769313486231570815e308;
                            else if (rsq > cutoffsq) vlj = 0.0;
                            else {
                                double div = siguv6 / (rsq * rsq * rsq);
                                vlj = 4.0 * epsuv * div * (div - 1.0);
                            }
                            if (only_origin) {
                                for (int k = 0; k < no; ++k) v[k] = v[k] + vlj;
                                break;
                            }
                            v[io] = v[io] + vlj;
                        }
                    }
                }
            }
        }
    }
    free(tab);
    /* vext_total_sum: add vextq, clip at qfact/2, reject NaN/Inf */
    const double thr = QFACT / 2.0;
    for (long i = 0; i < N * no; ++i) {
        double v = vext[i];
        if (vextq) v = v + vextq[i];
        if (v > thr) v = thr;
        if (v != v || isinf(v)) { set_err("NaN/Inf in vext"); free(vextq); return -1; }
        vext[i] = v;
    }
    /* module_vext.f90:79-83 */
    for (long i = 0; i < N * no; ++i)
        if (vext[i] <= -thr) { set_err("vext below -threshold"); free(vextq); return -1; }
    free(vextq);
    if (lj_corr_out) *lj_corr_out = ljcorr;
    return 0;
}

/* mv_solute_to_center: module_solute.f90:146-187 */
void orc_center_solute(const orc *o, int nsol, double *xyz, int translate)
{
    const double L[3] = {o->lx, o->ly, o->lz};
    if (translate) {
        double mean[3] = {0, 0, 0};
        for (int s = 0; s < nsol; ++s) for (int d = 0; d < 3; ++d) mean[d] += xyz[3 * s + d];
        for (int d = 0; d < 3; ++d) mean[d] /= (double)nsol;
        for (int s = 0; s < nsol; ++s)
            for (int d = 0; d < 3; ++d) xyz[3 * s + d] = xyz[3 * s + d] + L[d] / 2.0 - mean[d];
    }
    for (int s = 0; s < nsol; ++s)
        for (int d = 0; d < 3; ++d) {
            double v = fmod(xyz[3 * s + d], L[d]);
            if (v < 0) v += L[d];
            xyz[3 * s + d] = v;
        }
}

/* guess_density: module_density.f90:267-284 */
int orc_guess_density(const orc *o, double *xi)
{
    double vextmax = (-log(EPSDP) - (double)0.05f) * o->kT;
    for (long i = 0; i < o->N * o->no; ++i) xi[i] = (o->vext[i] >= vextmax) ? 0.0 : 1.0;
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Moré-Thuente line search: module_lbfgs_nocedal_mdft.f90:1653-1959.         */
typedef struct {
    int brackt, stage;
    double ginit, gtest, gx, gy, finit, fx, fy, stx, sty, stmin, stmax, width, width1;
} ls_state;

enum { LS_FG = 0, LS_CONV = 1, LS_WARN = 2, LS_ERROR = 3 };

static void dcstep(double *stx, double *fx, double *dx, double *sty, double *fy, double *dy, double *stp,
                   double fp, double dp, int *brackt, double stpmin, double stpmax)
{
    const double p66 = (double)0.66f, two = 2.0, three = 3.0, zero = 0.0;
    double gamma, p, q, r, s, sgnd, stpc, stpf, stpq, theta;
    sgnd = dp * (*dx / fabs(*dx));
    if (fp > *fx) {
        theta = three * (*fx - fp) / (*stp - *stx) + *dx + dp;
        s = fmax(fmax(fabs(theta), fabs(*dx)), fabs(dp));
        gamma = s * sqrt((theta / s) * (theta / s) - (*dx / s) * (dp / s));
        if (*stp < *stx) gamma = -gamma;
        p = (gamma - *dx) + theta;
        q = ((gamma - *dx) + gamma) + dp;
        r = p / q;
        stpc = *stx + r * (*stp - *stx);
        stpq = *stx + ((*dx / ((*fx - fp) / (*stp - *stx) + *dx)) / two) * (*stp - *stx);
        if (fabs(stpc - *stx) < fabs(stpq - *stx)) stpf = stpc;
        else stpf = stpc + (stpq - stpc) / two;
        *brackt = 1;
    } else if (sgnd < zero) {
        theta = three * (*fx - fp) / (*stp - *stx) + *dx + dp;
        s = fmax(fmax(fabs(theta), fabs(*dx)), fabs(dp));
        gamma = s * sqrt((theta / s) * (theta / s) - (*dx / s) * (dp / s));
        if (*stp > *stx) gamma = -gamma;
        p = (gamma - dp) + theta;
        q = ((gamma - dp) + gamma) + *dx;
        r = p / q;
        stpc = *stp + r * (*stx - *stp);
        stpq = *stp + (dp / (dp - *dx)) * (*stx - *stp);
        if (fabs(stpc - *stp) > fabs(stpq - *stp)) stpf = stpc;
        else stpf = stpq;
        *brackt = 1;
    } else if (fabs(dp) < fabs(*dx)) {
        theta = three * (*fx - fp) / (*stp - *stx) + *dx + dp;
        s = fmax(fmax(fabs(theta), fabs(*dx)), fabs(dp));
        gamma = s * sqrt(fmax(zero, (theta / s) * (theta / s) - (*dx / s) * (dp / s)));
        if (*stp > *stx) gamma = -gamma;
        p = (gamma - dp) + theta;
        q = (gamma + (*dx - dp)) + gamma;
        r = p / q;
        if (r < zero && gamma != zero) stpc = *stp + r * (*stx - *stp);
        else if (*stp > *stx) stpc = stpmax;
        else stpc = stpmin;
        stpq = *stp + (dp / (dp - *dx)) * (*stx - *stp);
        if (*brackt) {
            if (fabs(stpc - *stp) < fabs(stpq - *stp)) stpf = stpc;
            else stpf = stpq;
            if (*stp > *stx) stpf = fmin(*stp + p66 * (*sty - *stp), stpf);
            else stpf = fmax(*stp + p66 * (*sty - *stp), stpf);
        } else {
            if (fabs(stpc - *stp) > fabs(stpq - *stp)) stpf = stpc;
            else stpf = stpq;
            stpf = fmin(stpmax, stpf);
            stpf = fmax(stpmin, stpf);
        }
    } else {
        if (*brackt) {
            theta = three * (fp - *fy) / (*sty - *stp) + *dy + dp;
            s = fmax(fmax(fabs(theta), fabs(*dy)), fabs(dp));
            gamma = s * sqrt((theta / s) * (theta / s) - (*dy / s) * (dp / s));
            if (*stp > *sty) gamma = -gamma;
            p = (gamma - dp) + theta;
            q = ((gamma - dp) + gamma) + *dy;
            r = p / q;
            stpc = *stp + r * (*sty - *stp);
            stpf = stpc;
        } else if (*stp > *stx) stpf = stpmax;
        else stpf = stpmin;
    }
    if (fp > *fx) { *sty = *stp; *fy = fp; *dy = dp; }
    else {
        if (sgnd < zero) { *sty = *stx; *fy = *fx; *dy = *dx; }
        *stx = *stp; *fx = fp; *dx = dp;
    }
    *stp = stpf;
}

static int dcsrch(double f, double g, double *stp, double ftol, double gtol, double xtol, double stpmin,
                  double stpmax, int start, ls_state *S)
{
    const double zero = 0.0, p5 = 0.5, p66 = (double)0.66f, xtrapl = (double)1.1f, xtrapu = 4.0;
    if (start) {
        if (*stp < stpmin || *stp > stpmax || g >= zero || ftol < zero || gtol < zero || xtol < zero ||
            stpmin < zero || stpmax < stpmin)
            return LS_ERROR;
        S->brackt = 0; S->stage = 1; S->finit = f; S->ginit = g; S->gtest = ftol * S->ginit;
        S->width = stpmax - stpmin; S->width1 = S->width / p5;
        S->stx = zero; S->fx = S->finit; S->gx = S->ginit;
        S->sty = zero; S->fy = S->finit; S->gy = S->ginit;
        S->stmin = zero; S->stmax = *stp + xtrapu * *stp;
        return LS_FG;
    }
    int task = LS_FG;
    double ftest = S->finit + *stp * S->gtest;
    if (S->stage == 1 && f <= ftest && g >= zero) S->stage = 2;
    if (S->brackt && (*stp <= S->stmin || *stp >= S->stmax)) task = LS_WARN;
    if (S->brackt && S->stmax - S->stmin <= xtol * S->stmax) task = LS_WARN;
    if (*stp == stpmax && f <= ftest && g <= S->gtest) task = LS_WARN;
    if (*stp == stpmin && (f > ftest || g >= S->gtest)) task = LS_WARN;
    if (f <= ftest && fabs(g) <= gtol * (-S->ginit)) task = LS_CONV;
    if (task == LS_WARN || task == LS_CONV) return task;
    if (S->stage == 1 && f <= S->fx && f > ftest) {
        double fm = f - *stp * S->gtest, fxm = S->fx - S->stx * S->gtest, fym = S->fy - S->sty * S->gtest;
        double gm = g - S->gtest, gxm = S->gx - S->gtest, gym = S->gy - S->gtest;
        dcstep(&S->stx, &fxm, &gxm, &S->sty, &fym, &gym, stp, fm, gm, &S->brackt, S->stmin, S->stmax);
        S->fx = fxm + S->stx * S->gtest; S->fy = fym + S->sty * S->gtest;
        S->gx = gxm + S->gtest; S->gy = gym + S->gtest;
    } else {
        dcstep(&S->stx, &S->fx, &S->gx, &S->sty, &S->fy, &S->gy, stp, f, g, &S->brackt, S->stmin, S->stmax);
    }
    if (S->brackt) {
        if (fabs(S->sty - S->stx) >= p66 * S->width1) *stp = S->stx + p5 * (S->sty - S->stx);
        S->width1 = S->width;
        S->width = fabs(S->sty - S->stx);
    }
    if (S->brackt) { S->stmin = fmin(S->stx, S->sty); S->stmax = fmax(S->stx, S->sty); }
    else { S->stmin = *stp + xtrapl * (*stp - S->stx); S->stmax = *stp + xtrapu * (*stp - S->stx); }
    *stp = fmax(*stp, stpmin);
    *stp = fmin(*stp, stpmax);
    if ((S->brackt && (*stp <= S->stmin || *stp >= S->stmax)) || (S->brackt && S->stmax - S->stmin <= xtol * S->stmax))
        *stp = S->stx;
    return LS_FG;
}

/* ------------------------------------------------------------------------- */
/* Unconstrained L-BFGS-B driver: module_lbfgs_nocedal_mdft.f90:136-534 with */
/* energy_minimization.f90:232-290.  For an unconstrained problem the        */
/* compact-form step (formk/cmprlb/subsm) equals the two-loop recursion with */
/* H0 = I/theta; the two-loop form is used here.  Cauchy with no bounds and  */
/* col=0 gives z = x - g/theta.                                               */
static double ddot_(long n, const double *a, const double *b)
{
    double part[ORC_NCHUNK];
#pragma omp parallel for
    for (int ch = 0; ch < ORC_NCHUNK; ++ch) {
        double s = 0;
        for (long i = n * ch / ORC_NCHUNK; i < n * (ch + 1) / ORC_NCHUNK; ++i) s += a[i] * b[i];
        part[ch] = s;
    }
    double s = 0;
    for (int ch = 0; ch < ORC_NCHUNK; ++ch) s += part[ch];
    return s;
}
static double amax_(long n, const double *a)
{
    double s = 0;
    for (long i = 0; i < n; ++i) s = fmax(s, fabs(a[i]));
    return s;
}

/* The objective of a minimisation: F and its gradient at x (vectors of n). */
typedef int (*objective_fn)(void *ctx, const double *x, double *f, double *g);

static int lbfgs_core(objective_fn eval, void *ctx, long n, double *x, int m, double pgtol, double tol, int itermax,
                      double *f_out, int *nfg_out, int *iter_out, int *status_out);

static int single_objective(void *ctx, const double *x, double *f, double *g)
{
    return orc_energy_grad((orc *)ctx, x, f, g, NULL);
}

/* result: status 0=pgtol convergence, 1=f-reduction convergence, 2=abnormal line search, 3=itermax */
int orc_minimize(orc *o, double *x, int m, double pgtol, double tol, int itermax, double *f_out, int *nfg_out,
                 int *iter_out, int *status_out)
{
    return lbfgs_core(single_objective, o, o->N * o->no, x, m, pgtol, tol, itermax, f_out, nfg_out, iter_out, status_out);
}

typedef struct { orc *const *sp; int ns; const double *x; } mixture_ctx;

static int mixture_objective(void *ctx, const double *x, double *f, double *g)
{
    const mixture_ctx *c = (const mixture_ctx *)ctx;
    return orc_mixture_energy_grad(c->sp, c->ns, c->x, x, f, g, NULL);
}

/* The same L-BFGS over every species' xi at once, x = [ns][N][no] (energy_minimization's
   vector of all species). */
int orc_mixture_minimize(orc *const *sp, int ns, const double *xfrac, double *x, int m, double pgtol, double tol, int itermax,
                         double *f_out, int *nfg_out, int *iter_out, int *status_out)
{
    mixture_ctx c = {sp, ns, xfrac};
    return lbfgs_core(mixture_objective, &c, sp[0]->N * sp[0]->no * ns, x, m, pgtol, tol, itermax, f_out, nfg_out, iter_out,
                      status_out);
}

/* L-BFGS-B without bounds: module_lbfgs_nocedal_mdft.f90:136-534 (mainlb), the compact
   update of :1287-1318 and the line search of :1653-1959. */
static int lbfgs_core(objective_fn eval, void *ctx, long n, double *x, int m, double pgtol, double tol, int itermax,
                      double *f_out, int *nfg_out, int *iter_out, int *status_out)
{
    double *g = malloc(sizeof(double) * n), *d = malloc(sizeof(double) * n), *t = malloc(sizeof(double) * n);
    double *r = malloc(sizeof(double) * n), *z = malloc(sizeof(double) * n);
    double *S = malloc(sizeof(double) * n * m), *Y = malloc(sizeof(double) * n * m);
    double *rhos = malloc(sizeof(double) * m), *alph = malloc(sizeof(double) * m);
    const double epsmch = EPSDP;
    const double ftol = (double)0.001f, gtol = (double)0.9f, xtol = (double)0.1f, big = 1.0 + 10;
    double f, fold = 0, theta = 1.0, stp = 0, gd = 0, gdold = 0, dtd, dnorm, stpmx;
    int col = 0, head = 0, itail = 0, iupdat = 0, iter = 0, nfgv = 0, status = 3;
    if (eval(ctx, x, &f, g)) goto fail;
    nfgv = 1;
    double sbgnrm = amax_(n, g);
    if (sbgnrm <= pgtol) { status = 0; goto done; }
    while (iter < itermax) {
        /* direction */
        if (col == 0) {
            for (long i = 0; i < n; ++i) z[i] = x[i] - g[i] / theta;
        } else {
            for (long i = 0; i < n; ++i) d[i] = -g[i];
            for (int k = col - 1; k >= 0; --k) {
                int j = (head + k) % m;
                alph[j] = rhos[j] * ddot_(n, S + (long)j * n, d);
#pragma omp parallel for
                for (long i = 0; i < n; ++i) d[i] -= alph[j] * Y[(long)j * n + i];
            }
            for (long i = 0; i < n; ++i) d[i] /= theta;
            for (int k = 0; k < col; ++k) {
                int j = (head + k) % m;
                double beta = rhos[j] * ddot_(n, Y + (long)j * n, d);
#pragma omp parallel for
                for (long i = 0; i < n; ++i) d[i] += (alph[j] - beta) * S[(long)j * n + i];
            }
            for (long i = 0; i < n; ++i) z[i] = x[i] + d[i];
        }
        for (long i = 0; i < n; ++i) d[i] = z[i] - x[i];
        /* lnsrlb */
        dtd = ddot_(n, d, d);
        dnorm = sqrt(dtd);
        stpmx = big;
        stp = (iter == 0) ? fmin(1.0 / dnorm, stpmx) : 1.0;
        memcpy(t, x, sizeof(double) * n);
        memcpy(r, g, sizeof(double) * n);
        fold = f;
        int ifun = 0, iback = 0, info = 0, lstask;
        ls_state LS;
        int start = 1;
        for (;;) {
            gd = ddot_(n, g, d);
            if (ifun == 0) {
                gdold = gd;
                if (gd >= 0.0) { info = -4; break; }
            }
            lstask = dcsrch(f, gd, &stp, ftol, gtol, xtol, 0.0, stpmx, start, &LS);
            start = 0;
            if (lstask == LS_ERROR) { info = -1; break; }
            if (lstask == LS_CONV || lstask == LS_WARN) break;
            ++ifun; ++nfgv; iback = ifun - 1;
            if (iback >= 20) break;
            if (stp == 1.0) memcpy(x, z, sizeof(double) * n);
            else for (long i = 0; i < n; ++i) x[i] = stp * d[i] + t[i];
            if (eval(ctx, x, &f, g)) goto fail;
        }
        if (info != 0 || iback >= 20) {
            memcpy(x, t, sizeof(double) * n);
            memcpy(g, r, sizeof(double) * n);
            f = fold;
            if (col == 0) { status = 2; ++iter; goto done; }
            col = 0; head = 0; itail = 0; theta = 1.0; iupdat = 0;
            continue;
        }
        ++iter;
        sbgnrm = amax_(n, g);
        if (sbgnrm <= pgtol) { status = 0; goto done; }
        if ((fold - f) <= tol) { status = 1; goto done; }
        for (long i = 0; i < n; ++i) r[i] = g[i] - r[i];
        double rr = ddot_(n, r, r), dr, ddum;
        if (stp == 1.0) { dr = gd - gdold; ddum = -gdold; }
        else { dr = (gd - gdold) * stp; for (long i = 0; i < n; ++i) d[i] *= stp; ddum = -gdold * stp; }
        if (dr <= epsmch * ddum) continue; /* skip the update */
        ++iupdat; /* matupd: module_lbfgs_nocedal_mdft.f90:1287-1318 */
        if (iupdat <= m) { col = iupdat; itail = (head + iupdat - 1) % m; }
        else { itail = (itail + 1) % m; head = (head + 1) % m; }
        memcpy(S + (long)itail * n, d, sizeof(double) * n);
        memcpy(Y + (long)itail * n, r, sizeof(double) * n);
        rhos[itail] = 1.0 / dr;
        theta = rr / dr;
    }
done:
    *f_out = f;
    *nfg_out = nfgv;
    *iter_out = iter;
    *status_out = status;
    free(g); free(d); free(t); free(r); free(z); free(S); free(Y); free(rhos); free(alph);
    return 0;
fail:
    free(g); free(d); free(t); free(r); free(z); free(S); free(Y); free(rhos); free(alph);
    return -1;
}

/* ------------------------------------------------------------------------- */
/* Pressure correction and the solvation free energy:                        */
/* module_pressure_correction.f90:7-156.  out = {dG, PMV, Pbulk, deltaN}     */
int orc_pressure_correction(orc *o, const double *xi, double ftot, double lj_corr, double *out)
{
    const long N = o->N;
    const int no = o->no;
    /* density integrated over orientations; Kahan sum stands in for sum_byfft_3d */
    double s = 0, comp = 0;
    for (long r = 0; r < N; ++r) {
        double dens = 0;
        for (int io = 0; io < no; ++io) {
            double x = xi[r * no + io];
            dens += x * x * o->rho0 * o->w[io];
        }
        double y = dens - comp, t = s + y;
        comp = (t - s) - y;
        s = t;
    }
    double nwith = s * o->dv;
    double nwithout = o->n0 * (o->lx * o->ly * o->lz);
    double deltaN = nwithout - nwith;
    double *zero = calloc((size_t)N * no, sizeof(double));
    double save = o->const_corr, f0;
    o->const_corr = 0.0;
    int rc = orc_energy_grad(o, zero, &f0, NULL, NULL);
    o->const_corr = save;
    free(zero);
    if (rc) return -1;
    double pbulk = f0 / (o->lx * o->ly * o->lz);
    double pmv = -deltaN / o->n0 * pbulk;
    out[0] = ftot + pmv + lj_corr;
    out[1] = pmv;
    out[2] = pbulk;
    out[3] = deltaN;
    return 0;
}
