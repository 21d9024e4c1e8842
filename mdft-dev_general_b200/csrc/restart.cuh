// The reference's density file: output/density.bin written after a solve
// (src/module_postprocessing.f90:45-95) and read back as a restart point
// (read_restart_file, src/module_density.f90:61-261).  Included by solve.cuh.
//
// File: Fortran unformatted sequential records, each framed by its 4-byte length before and
// after (gfortran's default).  Records: ns (negative when the full density follows), mmax,
// no, np, (nx, ny, nz), (dx, dy, dz), nsite, one record per solute site (the derived type
// site_type of src/module_system.f90:7-13 written component by component: name(100),
// type, n_sites, r(3), q, sig, eps, lambda1, lambda2, Z: 176 bytes), then for every grid
// point (x fastest) either one record of np complex projections angl2proj(xi(:, point)),
// or, for the full density, no records of one real each.
//
// Reading: the projections become xi on the file's grid (proj2angl with this handle's
// orientations, so mmax may grow), and that field is interpolated onto this handle's grid
// with the file's box centred in this one.  The reference loops over io, then over the
// file's cells (z, y, x, each from 1 to n-1) and writes every new point inside a cell, so a
// point on a cell face takes the value of the last cell that holds it, and points outside
// every cell keep their value.  That last cell is found per axis; the interpolation runs on
// the device, one thread per (point, orientation), with the reference's operation order
// and no fused multiply-adds.
#pragma once

#include <cstdint>
#include <cstdio>
#include <new>

namespace {

// p[pt][ip] = sum_io xi[pt][io] A[io][ip]  (A: [no][2 np], re/im interleaved)
__global__ void k_angl2proj_pts(const double *__restrict__ xi, const double *__restrict__ A, double2 *__restrict__ p, int no, int np,
                                long long N) {
    const long long n = N * np;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long pt = i / np;
        const int ip = (int)(i - pt * np);
        const double *x = xi + pt * no;
        double re = 0.0, im = 0.0;
        for (int io = 0; io < no; ++io) {
            re += x[io] * A[(size_t)io * 2 * np + 2 * ip];
            im += x[io] * A[(size_t)io * 2 * np + 2 * ip + 1];
        }
        p[i] = make_double2(re, im);
    }
}

// xi[pt][io] = sum_ip Re p B[2ip][io] + Im p B[2ip+1][io]  (proj2angl with the mu >= 0 half)
__global__ void k_proj2angl_pts(const double2 *__restrict__ p, const double *__restrict__ B, double *__restrict__ xi, int no, int np,
                                long long N) {
    const long long n = N * no;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long pt = i / no;
        const int io = (int)(i - pt * no);
        const double2 *q = p + pt * np;
        double s = 0.0;
        for (int ip = 0; ip < np; ++ip) s += q[ip].x * B[(size_t)(2 * ip) * no + io] + q[ip].y * B[(size_t)(2 * ip + 1) * no + io];
        xi[i] = s;
    }
}

struct RegridArgs {
    int nx, ny, nz, no;           // this grid
    int px, py, pz;               // the file's grid
    const int *cell[3];           // per axis and new index: the last file cell (0-based) holding it, or -1
    const double *w[3];           // its interpolation weight (x - x0)/(x1 - x0)
};

__device__ __forceinline__ double lerp_rn(double a, double b, double t) {
    // a (1 - t) + b t, rounded step by step as the reference's expression
    return __dadd_rn(__dmul_rn(a, __dadd_rn(1.0, -t)), __dmul_rn(b, t));
}

__global__ void k_restart_regrid(const double *__restrict__ xp, double *__restrict__ xi, RegridArgs a) {
    const long long N = (long long)a.nx * a.ny * a.nz;
    const long long n = N * a.no;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long pt = i / a.no;
        const int io = (int)(i - pt * a.no);
        const int ix = (int)(pt % a.nx);
        const long long t = pt / a.nx;
        const int iy = (int)(t % a.ny), iz = (int)(t / a.ny);
        const int cx = a.cell[0][ix], cy = a.cell[1][iy], cz = a.cell[2][iz];
        if (cx < 0 || cy < 0 || cz < 0) continue;
        const double xd = a.w[0][ix], yd = a.w[1][iy], zd = a.w[2][iz];
        auto at = [&](int x, int y, int z) { return xp[(((long long)z * a.py + y) * a.px + x) * a.no + io]; };
        const double xi00 = lerp_rn(at(cx, cy, cz), at(cx + 1, cy, cz), xd);
        const double xi01 = lerp_rn(at(cx, cy, cz + 1), at(cx + 1, cy, cz + 1), xd);
        const double xi10 = lerp_rn(at(cx, cy + 1, cz), at(cx + 1, cy + 1, cz), xd);
        const double xi11 = lerp_rn(at(cx, cy + 1, cz + 1), at(cx + 1, cy + 1, cz + 1), xd);
        const double xi0 = lerp_rn(xi00, xi10, yd);
        const double xi1 = lerp_rn(xi01, xi11, yd);
        xi[i] = lerp_rn(xi0, xi1, zd);
    }
}

// Per axis: for every new index (0-based) the last file cell, in the reference's loop
// order, whose [x0, x1] holds it (src/module_density.f90:204-214), with its weight.
void regrid_axis(int n, double d, int np_, double dp, double off, std::vector<int> &cell, std::vector<double> &w) {
    cell.assign(n, -1);
    w.assign(n, 0.0);
    for (int k = 1; k <= np_ - 1; ++k) {
        const double x0 = (k - 1) * dp + off, x1 = k * dp + off;
        // node range in double, clamped to [0, n+1] before the conversion to int
        const double flo = std::ceil(x0 / d + 1), fhi = std::floor(x1 / d + 1);
        const int lo = std::max(1, (int)std::min<double>(std::max<double>(flo, 0.0), n + 1.0));
        const int hi = std::min(n, (int)std::min<double>(std::max<double>(fhi, 0.0), n + 1.0));
        for (int i = lo; i <= hi; ++i) {
            const double x = (i - 1) * d;
            cell[i - 1] = k - 1;
            w[i - 1] = (x - x0) / (x1 - x0);
        }
    }
}

// Fortran unformatted sequential records (4-byte length markers)
struct FRecWriter {
    FILE *f;
    bool ok = true;
    void rec(const void *p, uint32_t n) {
        ok = ok && std::fwrite(&n, 4, 1, f) == 1 && (n == 0 || std::fwrite(p, n, 1, f) == 1) && std::fwrite(&n, 4, 1, f) == 1;
    }
};

struct FRecReader {
    FILE *f;
    std::string err;
    // one record into buf; false (with err) at a short read or a mismatched frame
    bool rec(std::vector<unsigned char> &buf) {
        uint32_t n = 0, m = 0;
        if (std::fread(&n, 4, 1, f) != 1) { err = "unexpected end of file"; return false; }
        if (n > (1u << 20)) { err = "record longer than any of this format"; return false; }  // <= 16 np bytes
        buf.resize(n);
        if (n && std::fread(buf.data(), n, 1, f) != 1) { err = "truncated record"; return false; }
        if (std::fread(&m, 4, 1, f) != 1 || m != n) { err = "record markers do not match"; return false; }
        return true;
    }
};

constexpr uint32_t kSiteRecord = 176;

void pack_site(unsigned char *o, double x, double y, double z, double q, double sig, double eps, int Z) {
    std::memset(o, ' ', 100);                 // name
    const int32_t zero = 0, z32 = Z;
    std::memcpy(o + 100, &zero, 4);           // type
    std::memcpy(o + 104, &zero, 4);           // n_sites
    const double v[8] = {x, y, z, q, sig, eps, 0.0, 0.0};  // r(3), q, sig, eps, lambda1, lambda2
    std::memcpy(o + 108, v, 64);
    std::memcpy(o + 172, &z32, 4);            // Z
}

}  // namespace

extern "C" {

int mdft_write_density_bin(mdft_handle *h, const double *xi, int nsite, const double *q, const double *sig, const double *eps,
                           const double *xyz, const int *Z, int full, const char *path) {
    if (!h || !path || nsite < 0 || (nsite > 0 && (!q || !sig || !eps || !xyz))) { set_error("null or invalid argument"); return MDFT_E_ARG; }
    const Grid &g = h->g;
    const size_t nf = (size_t)g.N * g.no;
    int rc;
    const double *dx = nullptr;
    if (xi) {
        if ((rc = check_cuda(cudaMemcpyAsync(h->xi.p, xi, nf * 8, cudaMemcpyHostToDevice, h->stream), "xi upload"))) return rc;
        dx = h->xi.p;
    } else {
        if (!h->lb.x.p) { set_error("no solve has run on this handle"); return MDFT_E_STATE; }
        dx = h->lb.x.p;
    }
    std::vector<double> hx;
    std::vector<double2> hp;
    if (full) {
        hx.resize(nf);
        if ((rc = check_cuda(cudaMemcpyAsync(hx.data(), dx, nf * 8, cudaMemcpyDeviceToHost, h->stream), "xi download"))) return rc;
    } else {
        DevBuf<double2> p;
        const size_t n = (size_t)g.N * g.np;
        if ((rc = alloc_check(p.alloc(n), "projections", n * 16))) return rc;
        k_angl2proj_pts<<<vec_grid(), 256, 0, h->stream>>>(dx, h->A.p, p.p, g.no, g.np, g.N);
        h->launches += 1;
        hp.resize(n);
        if ((rc = check_cuda(cudaMemcpyAsync(hp.data(), p.p, n * 16, cudaMemcpyDeviceToHost, h->stream), "projections download"))) return rc;
        if ((rc = check_cuda(cudaStreamSynchronize(h->stream), "angl2proj"))) return rc;
    }
    if ((rc = check_cuda(cudaStreamSynchronize(h->stream), "density download"))) return rc;
    FILE *f = std::fopen(path, "wb");
    if (!f) { set_error("cannot create %s", path); return MDFT_E_IO; }
    FRecWriter w{f};
    const int32_t ns = full ? -1 : 1, mmax = g.mmax, no = g.no, np = g.np, n3[3] = {g.nx, g.ny, g.nz}, ns32 = nsite;
    const double d3[3] = {g.dx, g.dy, g.dz};
    w.rec(&ns, 4);
    w.rec(&mmax, 4);
    w.rec(&no, 4);
    w.rec(&np, 4);
    w.rec(n3, 12);
    w.rec(d3, 24);
    w.rec(&ns32, 4);
    unsigned char site[kSiteRecord];
    for (int s = 0; s < nsite; ++s) {
        pack_site(site, xyz[3 * s], xyz[3 * s + 1], xyz[3 * s + 2], q[s], sig[s], eps[s], Z ? Z[s] : 0);
        w.rec(site, kSiteRecord);
    }
    if (full) {
        for (size_t i = 0; i < nf && w.ok; ++i) w.rec(&hx[i], 8);
    } else {
        for (long long pt = 0; pt < g.N && w.ok; ++pt) w.rec(&hp[(size_t)pt * g.np], (uint32_t)(16 * g.np));
    }
    const bool ok = w.ok && std::fclose(f) == 0;
    if (!ok) { set_error("writing %s failed", path); return MDFT_E_IO; }
    return MDFT_OK;
}

int mdft_read_density_bin(mdft_handle *h, const char *path, int nsite, const double *sig, const double *eps, const double *xyz,
                          double *xi) {
    if (!h || !path || !xi || nsite < 0 || (nsite > 0 && (!sig || !eps || !xyz))) { set_error("null or invalid argument"); return MDFT_E_ARG; }
    const Grid &g = h->g;
    FILE *f = std::fopen(path, "rb");
    if (!f) { set_error("restart file %s not found", path); return MDFT_E_IO; }
    struct Closer { FILE *f; ~Closer() { std::fclose(f); } } closer{f};
    FRecReader r{f};
    std::vector<unsigned char> b;
    auto rd_ints = [&](int32_t *v, int n) -> bool {
        if (!r.rec(b)) return false;
        if (b.size() != 4u * n) { r.err = "header record of unexpected length"; return false; }
        std::memcpy(v, b.data(), 4u * n);
        return true;
    };
    int32_t ns, mmax_p, no_p, np_p, n3[3], nsite_p;
    double d3[3];
    bool ok = rd_ints(&ns, 1) && rd_ints(&mmax_p, 1) && rd_ints(&no_p, 1) && rd_ints(&np_p, 1) && rd_ints(n3, 3);
    if (ok && r.rec(b)) {
        if (b.size() != 24) { r.err = "grid spacing record of unexpected length"; ok = false; }
        else std::memcpy(d3, b.data(), 24);
    } else {
        ok = false;
    }
    ok = ok && rd_ints(&nsite_p, 1);
    if (!ok) { set_error("%s: %s", path, r.err.c_str()); return MDFT_E_IO; }
    const bool full = ns < 0;
    if ((full ? -ns : ns) != 1) { set_error("%s: %d solvent species (one is supported)", path, full ? -ns : ns); return MDFT_E_ARG; }
    if (n3[0] < 1 || n3[1] < 1 || n3[2] < 1 || n3[0] > 65536 || n3[1] > 65536 || n3[2] > 65536 || no_p < 1 || np_p < 1 ||
        (long long)n3[0] * n3[1] * n3[2] > (1LL << 33)) {
        set_error("%s: bad grid in header", path);
        return MDFT_E_IO;
    }
    for (int a = 0; a < 3; ++a)
        if (!(std::isfinite(d3[a]) && d3[a] > 0.0 && d3[a] * n3[a] <= 1.0e9)) {
            set_error("%s: bad grid spacing in header (%g)", path, d3[a]);
            return MDFT_E_IO;
        }
    // the file's box centred in this one (src/module_density.f90:129-131)
    const double off[3] = {(g.lx - d3[0] * n3[0]) / 2, (g.ly - d3[1] * n3[1]) / 2, (g.lz - d3[2] * n3[2]) / 2};
    if (nsite_p > nsite) { set_error("%s: %d solute sites in the file, %d given", path, nsite_p, nsite); return MDFT_E_ARG; }
    for (int s = 0; s < nsite_p; ++s) {  // :141-158 (a count mismatch alone is only reported there)
        if (!r.rec(b) || b.size() != kSiteRecord) { set_error("%s: site record %d: %s", path, s + 1, r.err.empty() ? "bad length" : r.err.c_str()); return MDFT_E_IO; }
        double v[6];
        std::memcpy(v, b.data() + 108, 48);
        if (xyz[3 * s] != v[0] + off[0] || xyz[3 * s + 1] != v[1] + off[1] || xyz[3 * s + 2] != v[2] + off[2] || sig[s] != v[4] ||
            eps[s] != v[5]) {
            set_error("%s: solute site %d differs from the file's", path, s + 1);
            return MDFT_E_ARG;
        }
    }
    const size_t nf = (size_t)g.N * g.no;
    int rc;
    if (full) {
        // read straight into this grid: the file must have this grid and orientations (:242-253)
        if (n3[0] != g.nx || n3[1] != g.ny || n3[2] != g.nz || no_p != g.no) {
            set_error("%s: a full-density file needs the same grid and orientations", path);
            return MDFT_E_ARG;
        }
        for (size_t i = 0; i < nf; ++i) {
            if (!r.rec(b) || b.size() != 8) { set_error("%s: density record %zu: %s", path, i, r.err.empty() ? "bad length" : r.err.c_str()); return MDFT_E_IO; }
            std::memcpy(&xi[i], b.data(), 8);
        }
        return MDFT_OK;
    }
    if (np_p > g.np) { set_error("%s: %d projections, this grid has %d (mmax %d < %d)", path, np_p, g.np, g.mmax, mmax_p); return MDFT_E_ARG; }
    const long long Np = (long long)n3[0] * n3[1] * n3[2];
    std::vector<double2> hp;
    try {
        hp.assign((size_t)Np * g.np, make_double2(0.0, 0.0));
    } catch (const std::bad_alloc &) {
        set_error("%s: no host memory for %lld points x %d projections", path, Np, g.np);
        return MDFT_E_NOMEM;
    }
    for (long long pt = 0; pt < Np; ++pt) {
        if (!r.rec(b) || b.size() != 16u * np_p) { set_error("%s: projection record %lld: %s", path, pt, r.err.empty() ? "bad length" : r.err.c_str()); return MDFT_E_IO; }
        std::memcpy(&hp[(size_t)pt * g.np], b.data(), 16u * np_p);
    }
    std::vector<int> cells[3];
    std::vector<double> ws[3];
    const int nn[3] = {g.nx, g.ny, g.nz};
    const double dd[3] = {g.dx, g.dy, g.dz};
    for (int a = 0; a < 3; ++a) regrid_axis(nn[a], dd[a], n3[a], d3[a], off[a], cells[a], ws[a]);
    DevBuf<double2> dp;
    DevBuf<double> dxp, dw[3];
    DevBuf<int> dc[3];
    if ((rc = alloc_check(dp.alloc(hp.size()), "file projections", hp.size() * 16))) return rc;
    if ((rc = alloc_check(dxp.alloc((size_t)Np * g.no), "file density", (size_t)Np * g.no * 8))) return rc;
    for (int a = 0; a < 3; ++a) {
        if ((rc = alloc_check(dc[a].alloc(nn[a]), "regrid cells", nn[a] * 4))) return rc;
        if ((rc = alloc_check(dw[a].alloc(nn[a]), "regrid weights", nn[a] * 8))) return rc;
        cudaMemcpyAsync(dc[a].p, cells[a].data(), nn[a] * 4, cudaMemcpyHostToDevice, h->stream);
        cudaMemcpyAsync(dw[a].p, ws[a].data(), nn[a] * 8, cudaMemcpyHostToDevice, h->stream);
    }
    cudaMemcpyAsync(dp.p, hp.data(), hp.size() * 16, cudaMemcpyHostToDevice, h->stream);
    if ((rc = check_cuda(cudaMemcpyAsync(h->xi.p, xi, nf * 8, cudaMemcpyHostToDevice, h->stream), "xi upload"))) return rc;
    k_proj2angl_pts<<<vec_grid(), 256, 0, h->stream>>>(dp.p, h->B.p, dxp.p, g.no, g.np, Np);
    RegridArgs ra{g.nx, g.ny, g.nz, g.no, n3[0], n3[1], n3[2], {dc[0].p, dc[1].p, dc[2].p}, {dw[0].p, dw[1].p, dw[2].p}};
    k_restart_regrid<<<vec_grid(), 256, 0, h->stream>>>(dxp.p, h->xi.p, ra);
    h->launches += 2;
    if ((rc = check_cuda(cudaMemcpyAsync(xi, h->xi.p, nf * 8, cudaMemcpyDeviceToHost, h->stream), "xi download"))) return rc;
    return check_cuda(cudaStreamSynchronize(h->stream), "restart");
}

}  // extern "C"
