// The MRSO rotational-invariant Ornstein-Zernike step in the local q-frame
// (S3-S5 of src/module_energy_cproj_mrso.f90:441-674), one warp per (q, -q)
// pair.  Per pair the warp builds the rotation matrices R^m_{mup,khi}(q) of
// src/module_rotation.f90:119-247 in shared memory, rotates both projection
// vectors into the q-frame, applies the linearly interpolated
// c^{mn}_{mu nu khi}(|q|), flushes tiny values, rotates back with conj(R) and
// writes both results in place.
//
// Pair bookkeeping: the reference walks iz_q = 1..nz/2+1 (all iy, ix) and
// skips a point whose pair is already done.  Planes kz=0 and kz=Nyquist hold
// both members of their pairs; the member reached first in (iy, ix) order is
// the one treated as q.  Here (0-based) a k-point with iz in [1, nz/2) is
// always the q of its pair; with iz in {0, nz/2} it is the q iff
// iy*nx+ix <= iym*nx+ixm.  A self-conjugate point (q == -q) ends with the -q
// result, conjugated when any index sits at Nyquist (:648-656).
#pragma once

#include "common.cuh"

namespace mdft {

constexpr int kRMax = 6;  // coefficient tables of src/module_rotation.f90:13-34 (mmax_max = 6)
constexpr int kRW = 2 * kRMax + 1;
constexpr int kMaxNpConst = 192;

struct RotCoef {
    double a[kRMax + 1][kRW][kRW];
    double b[kRMax + 1][kRW][kRW];
    double c[kRMax + 1][kRW];
    double d[kRMax + 1][kRW];
};

__constant__ RotCoef c_rot;
__constant__ int c_ia_start[kMaxNpConst];
__constant__ int c_pm[kMaxNpConst], c_pmup[kMaxNpConst], c_pmu2[kMaxNpConst];

inline void build_rot_coef(RotCoef &rc) {
    std::memset(&rc, 0, sizeof rc);
    auto sq = [](int k) { return k <= 0 ? 0.0 : std::sqrt((double)k); };
    const double sqrt2 = std::sqrt(2.0);
    for (int l = 2; l <= kRMax; ++l)
        for (int m = -l; m <= l; ++m) {
            for (int m1 = -l + 1; m1 <= l - 1; ++m1) {
                rc.a[l][m + kRMax][m1 + kRMax] = sq(l + m) * sq(l - m) / (sq(l + m1) * sq(l - m1));
                rc.b[l][m + kRMax][m1 + kRMax] = sq(l + m) * sq(l + m - 1) / (sqrt2 * sq(l + m1) * sq(l - m1));
            }
            rc.c[l][m + kRMax] = sqrt2 * sq(l + m) * sq(l - m) / (sq(2 * l) * sq(2 * l - 1));
            rc.d[l][m + kRMax] = sq(l + m) * sq(l + m - 1) / (sq(2 * l) * sq(2 * l - 1));
        }
}

struct OzArgs {
    int nx, ny, nz;
    long long N;
    int mmax, mrso, np, ncoef, nq;
    double dq;
    double twopi_lx, twopi_ly, twopi_lz;  // 2 pi / L
    int quirks;                           // 1: FP32 rounding of the flushed entries, as the reference
    long long nk;                         // k-points in the half space iz <= nz/2
};

__host__ __device__ inline int rot_off(int l) { return l * (4 * l * l - 1) / 3; }  // sum_{l'<l} (2l'+1)^2
__device__ __forceinline__ int ridx(int l, int m, int m1) { return rot_off(l) + (m + l) * (2 * l + 1) + (m1 + l); }

// ip of (m, mup, mu2) in the reference projection order
__device__ __forceinline__ int pidx(int m, int mup, int mu2, int mrso) {
    int off = 0;
    for (int k = 0; k < m; ++k) off += (2 * k + 1) * (k / mrso + 1);
    return off + (mup + m) * (m / mrso + 1) + mu2;
}

__device__ __forceinline__ double sp_round(double x, int quirks) { return quirks ? (double)__double2float_rn(x) : x; }

__device__ __forceinline__ double2 zmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 zmulc(double2 a, double2 b) {  // a * conj(b)
    return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}

// Rotation matrix R(q) into shared memory (packed), warp-cooperative.
__device__ void build_rotation(double2 *R, int mmax, double qx, double qy, double qz, int quirks) {
    const int lane = threadIdx.x & 31;
    if (mmax == 0) {
        if (lane == 0) R[0] = make_double2(1.0, 0.0);
        __syncwarp();
        return;
    }
    double r3[3], r2[3], r1[3];
    if (qx == 0.0 && qy == 0.0 && qz == 0.0) { r3[0] = 0; r3[1] = 0; r3[2] = 1; }
    else { r3[0] = qx; r3[1] = qy; r3[2] = qz; }
    if (r3[0] != 0.0 || r3[1] != 0.0) {  // z x r3
        r2[0] = -r3[1]; r2[1] = r3[0]; r2[2] = 0.0;
    } else {  // r3 x x
        r2[0] = 0.0; r2[1] = r3[2]; r2[2] = -r3[1];
    }
    double n3 = sqrt(r3[0] * r3[0] + r3[1] * r3[1] + r3[2] * r3[2]);
    double n2 = sqrt(r2[0] * r2[0] + r2[1] * r2[1] + r2[2] * r2[2]);
    for (int i = 0; i < 3; ++i) { r3[i] /= n3; r2[i] /= n2; }
    r1[0] = r2[1] * r3[2] - r2[2] * r3[1];
    r1[1] = r2[2] * r3[0] - r2[0] * r3[2];
    r1[2] = r2[0] * r3[1] - r2[1] * r3[0];
    // rmat(i,j) = r_j[i-1]
    const double sqrt2 = 1.4142135623730950488016887242097;
    if (lane == 0) R[0] = make_double2(1.0, 0.0);
    if (lane < 9) {
        const int m = lane / 3 - 1, m1 = lane % 3 - 1;
        double f = 0, g = 0;
        // src/module_rotation.f90:175-193
        if (m == -1 && m1 == -1) { f = (r2[1] + r1[0]) * 0.5; g = (r1[1] - r2[0]) * 0.5; }
        if (m == -1 && m1 == 0) { f = r3[0] / sqrt2; g = r3[1] / sqrt2; }
        if (m == -1 && m1 == 1) { f = (r2[1] - r1[0]) * 0.5; g = (-r1[1] - r2[0]) * 0.5; }
        if (m == 0 && m1 == -1) { f = r1[2] / sqrt2; g = -r2[2] / sqrt2; }
        if (m == 0 && m1 == 0) { f = r3[2]; g = 0.0; }
        if (m == 0 && m1 == 1) { f = -r1[2] / sqrt2; g = -r2[2] / sqrt2; }
        if (m == 1 && m1 == -1) { f = (r2[1] - r1[0]) * 0.5; g = (r1[1] + r2[0]) * 0.5; }
        if (m == 1 && m1 == 0) { f = -r3[0] / sqrt2; g = r3[1] / sqrt2; }
        if (m == 1 && m1 == 1) { f = (r2[1] + r1[0]) * 0.5; g = (r2[0] - r1[1]) * 0.5; }
        R[ridx(1, m, m1)] = make_double2(f, g);
    }
    __syncwarp();
    for (int l = 2; l <= mmax; ++l) {
        const int l1 = l - 1;
        const double2 p0 = R[ridx(1, 0, 0)], pp = R[ridx(1, 1, 0)], pm = R[ridx(1, -1, 0)];
        const double2 q0 = R[ridx(1, 0, 1)], qp = R[ridx(1, 1, 1)], qm = R[ridx(1, -1, 1)];
        const int ncomp = (l + 1) * (l + 1) + l * l;  // directly computed entries
        double2 val[2];
        int em[2], em1[2];
        int cnt = 0;
        for (int e = lane; e < ncomp; e += 32, ++cnt) {
            int m, m1;
            if (e < (l + 1) * (l + 1)) { m = -l + e / (l + 1); m1 = e % (l + 1); }      // m <= 0, m1 = 0..l
            else { int e2 = e - (l + 1) * (l + 1); m = 1 + e2 / l; m1 = 1 + e2 % l; }  // m > 0, m1 = 1..l
            double f, g;
            if (m1 < l) {
                if (m == -l) {
                    double bb = c_rot.b[l][-m + kRMax][m1 + kRMax];
                    double2 u = R[ridx(l1, m + 1, m1)];
                    f = bb * (pm.x * u.x - pm.y * u.y);
                    g = bb * (pm.x * u.y + pm.y * u.x);
                } else if (m == l) {
                    double bb = c_rot.b[l][m + kRMax][m1 + kRMax];
                    double2 u = R[ridx(l1, m - 1, m1)];
                    f = bb * (pp.x * u.x - pp.y * u.y);
                    g = bb * (pp.x * u.y + pp.y * u.x);
                } else {
                    double aa = c_rot.a[l][m + kRMax][m1 + kRMax];
                    double bp = c_rot.b[l][m + kRMax][m1 + kRMax], bmn = c_rot.b[l][-m + kRMax][m1 + kRMax];
                    double2 u0 = R[ridx(l1, m, m1)];
                    double2 up = (m - 1 >= -l1) ? R[ridx(l1, m - 1, m1)] : make_double2(0, 0);
                    double2 um = (m + 1 <= l1) ? R[ridx(l1, m + 1, m1)] : make_double2(0, 0);
                    f = aa * (p0.x * u0.x) + bp * (pp.x * up.x - pp.y * up.y) + bmn * (pm.x * um.x - pm.y * um.y);
                    g = aa * (p0.x * u0.y) + bp * (pp.x * up.y + pp.y * up.x) + bmn * (pm.x * um.y + pm.y * um.x);
                }
            } else {  // m1 == l
                if (m == -l) {
                    double dd = c_rot.d[l][-m + kRMax];
                    double2 u = R[ridx(l1, m + 1, m1 - 1)];
                    f = dd * (qm.x * u.x - qm.y * u.y);
                    g = dd * (qm.x * u.y + qm.y * u.x);
                } else if (m == l) {
                    double dd = c_rot.d[l][m + kRMax];
                    double2 u = R[ridx(l1, m - 1, m1 - 1)];
                    f = dd * (qp.x * u.x - qp.y * u.y);
                    g = dd * (qp.x * u.y + qp.y * u.x);
                } else {
                    double cc = c_rot.c[l][m + kRMax], dp = c_rot.d[l][m + kRMax], dmn = c_rot.d[l][-m + kRMax];
                    double2 u0 = R[ridx(l1, m, m1 - 1)];
                    double2 up = (m - 1 >= -l1) ? R[ridx(l1, m - 1, m1 - 1)] : make_double2(0, 0);
                    double2 um = (m + 1 <= l1) ? R[ridx(l1, m + 1, m1 - 1)] : make_double2(0, 0);
                    f = cc * (q0.x * u0.x - q0.y * u0.y) + dp * (qp.x * up.x - qp.y * up.y) + dmn * (qm.x * um.x - qm.y * um.y);
                    g = cc * (q0.x * u0.y + q0.y * u0.x) + dp * (qp.x * up.y + qp.y * up.x) + dmn * (qm.x * um.y + qm.y * um.x);
                }
            }
            val[cnt] = make_double2(f, g);
            em[cnt] = m;
            em1[cnt] = m1;
        }
        __syncwarp();
        for (int c = 0; c < cnt; ++c) {
            const int m = em[c], m1 = em1[c];
            const double s = neg1pow(m + m1);
            if (m == 0 && m1 == 0) {
                R[ridx(l, 0, 0)] = make_double2(val[c].x, -val[c].y);  // f kept, g negated by the fill
            } else {
                R[ridx(l, m, m1)] = val[c];
                R[ridx(l, -m, -m1)] = make_double2(s * val[c].x, -s * val[c].y);
            }
        }
        __syncwarp();
    }
    // src/module_energy_cproj_mrso.f90:491-492: flush |Re|,|Im| < epsilon(1.) (the other part
    // goes through Fortran's default-kind cmplx, i.e. FP32)
    for (int e = lane; e < rot_off(mmax + 1); e += 32) {
        double2 v = R[e];
        if (fabs(v.x) < kEpsSp) { v.x = 0.0; v.y = sp_round(v.y, quirks); }
        if (fabs(v.y) < kEpsSp) { v.x = sp_round(v.x, quirks); v.y = 0.0; }
        R[e] = v;
    }
    __syncwarp();
}

// smem per warp: R (rot_off(mmax+1)) + 6 np complex
__global__ void __launch_bounds__(256) k_oz_f64(double2 *__restrict__ planes, const double2 *__restrict__ ctab, OzArgs a) {
    extern __shared__ double2 oz_smem[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int nrot = rot_off(a.mmax + 1);
    const int np = a.np;
    double2 *R = oz_smem + (size_t)warp * (nrot + 6 * np);
    double2 *dq = R + nrot, *dmq = dq + np, *rq = dmq + np, *rmq = rq + np, *gq = rmq + np, *gmq = gq + np;
    const long long kk = (long long)blockIdx.x * (blockDim.x >> 5) + warp;
    if (kk >= a.nk) return;
    const int ix = (int)(kk % a.nx);
    const int iy = (int)((kk / a.nx) % a.ny);
    const int iz = (int)(kk / ((long long)a.nx * a.ny));
    const int ixm = (a.nx - ix) % a.nx, iym = (a.ny - iy) % a.ny, izm = (a.nz - iz) % a.nz;
    if (iz == 0 || 2 * iz == a.nz)
        if ((long long)iy * a.nx + ix > (long long)iym * a.nx + ixm) return;  // the partner is the q of this pair
    const bool selfconj = (ix == ixm && iy == iym && iz == izm);
    const bool nyq = (2 * ix == a.nx) || (2 * iy == a.ny) || (2 * iz == a.nz);
    const long long kq = ((long long)iz * a.ny + iy) * a.nx + ix;
    const long long kmq = ((long long)izm * a.ny + iym) * a.nx + ixm;
    // kproj (Nyquist positive): l-1 <= n/2 -> positive
    const double qx = (ix <= a.nx / 2 ? ix : ix - a.nx) * a.twopi_lx;
    const double qy = (iy <= a.ny / 2 ? iy : iy - a.ny) * a.twopi_ly;
    const double qz = (iz <= a.nz / 2 ? iz : iz - a.nz) * a.twopi_lz;
    for (int ip = lane; ip < np; ip += 32) {
        dq[ip] = planes[(size_t)ip * a.N + kq];
        dmq[ip] = planes[(size_t)ip * a.N + kmq];
    }
    build_rotation(R, a.mmax, qx, qy, qz, a.quirks);
    const int mrso = a.mrso;
    // rotation to the q-frame (:505-523)
    for (int o = lane; o < np; o += 32) {
        const int m = c_pm[o], khi = c_pmup[o], mu2 = c_pmu2[o];
        double2 s = make_double2(0, 0), t = make_double2(0, 0);
        const int base = pidx(m, -m, mu2, mrso), stride = m / mrso + 1;
        for (int mup = -m; mup <= m; ++mup) {
            const int jp = base + (mup + m) * stride;
            double2 r1 = R[ridx(m, mup, khi)], r2 = R[ridx(m, mup, -khi)];
            double2 u = zmul(dq[jp], r1), v = zmul(dmq[jp], r2);
            s.x += u.x; s.y += u.y;
            t.x += v.x; t.y += v.y;
        }
        rq[o] = s;
        const double sg = neg1pow(m);
        rmq[o] = make_double2(sg * t.x, sg * t.y);
    }
    __syncwarp();
    // interpolated c (:534-539) and OZ (:561-606)
    const double nrm = sqrt(qx * qx + qy * qy + qz * qz);
    const double eff = nrm / a.dq + 1.0;
    const int iq = (int)eff;
    const double alpha = eff - iq;
    const double2 *c0 = ctab + (size_t)(iq - 1) * a.ncoef;
    const double2 *c1 = ctab + (size_t)iq * a.ncoef;
    for (int ip = lane; ip < np; ip += 32) {
        const int khi = c_pmup[ip];
        int ia = c_ia_start[ip];
        double2 s = make_double2(0, 0), t = make_double2(0, 0);
        for (int n = abs(khi); n <= a.mmax; ++n) {
            const int nn = n / mrso;
            for (int nu2 = -nn; nu2 <= nn; ++nu2, ++ia) {
                double2 A = c0[ia], Bv = c1[ia];
                double2 ce = make_double2(alpha * Bv.x + (1.0 - alpha) * A.x, alpha * Bv.y + (1.0 - alpha) * A.y);
                double2 u, v;
                if (nu2 < 0) {
                    const int jp = pidx(n, khi, -nu2, mrso);
                    u = zmul(ce, rq[jp]);
                    v = zmul(ce, rmq[jp]);
                } else {
                    const int jp = pidx(n, khi, nu2, mrso);
                    u = zmulc(ce, rmq[jp]);
                    v = zmulc(ce, rq[jp]);
                }
                s.x += u.x; s.y += u.y;
                t.x += v.x; t.y += v.y;
            }
        }
        // underflow flush (:618-623)
        double2 *vv[2] = {&s, &t};
        for (int z = 0; z < 2; ++z) {
            double re = vv[z]->x, im = vv[z]->y;
            if (fabs(re) < kEpsDp && fabs(im) < kEpsDp) { re = 0.0; im = 0.0; }
            if (fabs(re) < kEpsDp) { re = 0.0; im = sp_round(im, a.quirks); }
            if (fabs(im) < kEpsDp) { re = sp_round(re, a.quirks); im = 0.0; }
            vv[z]->x = re;
            vv[z]->y = im;
        }
        gq[ip] = s;
        gmq[ip] = t;
    }
    __syncwarp();
    // back to the lab frame with conj(R) (:611-641) and store (:648-656)
    for (int o = lane; o < np; o += 32) {
        const int m = c_pm[o], mup = c_pmup[o], mu2 = c_pmu2[o];
        double2 s = make_double2(0, 0), t = make_double2(0, 0);
        const int base = pidx(m, -m, mu2, mrso), stride = m / mrso + 1;
        for (int khi = -m; khi <= m; ++khi) {
            const int jp = base + (khi + m) * stride;
            double2 u = zmulc(gq[jp], R[ridx(m, mup, khi)]);
            double2 v = zmulc(gmq[jp], R[ridx(m, mup, -khi)]);
            s.x += u.x; s.y += u.y;
            t.x += v.x; t.y += v.y;
        }
        const double sg = neg1pow(m);
        t.x *= sg;
        t.y *= sg;
        if (selfconj && nyq) t.y = -t.y;
        if (!selfconj) planes[(size_t)o * a.N + kq] = s;
        planes[(size_t)o * a.N + kmq] = t;
    }
}

inline size_t oz_smem_bytes(int mmax, int np, int warps) {
    return sizeof(double2) * (size_t)warps * (rot_off(mmax + 1) + 6 * np);
}

}  // namespace mdft
