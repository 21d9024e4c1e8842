// Rotated OZ step (S3-S5 of src/module_energy_cproj_mrso.f90:441-674), templated on the
// working precision T (double: parity path, float: mixed path).
//
// One warp per (q, -q) pair; a CTA takes W consecutive k-points (W = warps per CTA), so
// that the projections of the W points and of their W partners are read and written with
// coalesced accesses through shared memory.  Everything that depends only on (mmax, mrso)
// -- the term lists of the two rotations and of the OZ sum, and the recipe of the
// rotation-matrix recursion of src/module_rotation.f90:119-247 -- is precomputed on the
// host (OzTables) and staged in shared memory, so the per-pair work is table driven and
// free of divergent constant-memory reads.  Pairing, flushes and the Nyquist rule follow
// the reference (see k_oz.cuh).
#pragma once

#include <vector>

#include "common.cuh"
#include "k_fft.cuh"
#include "k_oz.cuh"

namespace mdft {

constexpr int kRecInts = 10;  // dest, fill, sign, special, (x, u) x 3
constexpr int kRecDbls = 3;   // coefficients

// Term encodings (one int per term): rotation terms jp | r1 << 8 | r2 << 19 (jp < 256,
// r < 2048); OZ terms ia | jp << 12 | direct << 20 (ia < 4096).  build_oz_tables checks the
// ranges.
__host__ __device__ inline int pack_rot_term(int jp, int r1, int r2) { return jp | (r1 << 8) | (r2 << 19); }
__host__ __device__ inline int pack_oz_term(int ia, int jp, int direct) { return ia | (jp << 12) | (direct << 20); }

struct OzTables {
    std::vector<int> ints;
    std::vector<double> dbls;
    int fwd_off = 0, fwd_terms = 0, oz_off = 0, oz_terms = 0, bwd_off = 0, bwd_terms = 0, sign = 0, lvl_off = 0,
        rec_int = 0;
    int nrot = 0;  // packed rotation entries; R[nrot] is a zero slot
};

// value = sum_t c_t X_t (x) U_t with X a level-1 entry and U a level l-1 entry (or the zero
// slot); R[dest] = value and R[fill] = (s Re, -s Im), except at (l,0,0) where the
// reference's symmetric fill negates Im in place.
// mix: the rotations of -q as the multi-species routine writes them, with R(m,mup,khi)
// (src/module_energy_cproj_mrso_mixture.f90:551,672) where the single-species routine uses
// R(m,mup,-khi) (src/module_energy_cproj_mrso.f90:517,636).  Only the r2 indices change.
inline bool build_oz_tables(const Grid &g, const CTable &ct, OzTables &T, bool mix = false) {
    const int M = g.mmax, mrso = g.mrso, np = g.np;
    if (np >= 256 || rot_off(M + 1) + 1 >= 2048 || ct.ncoef >= 4096) return false;  // term encodings
    auto pidx = [&](int m, int mup, int mu2) { return g.pidx(m, mup, mu2); };
    auto ridx = [](int l, int m, int m1) { return rot_off(l) + (m + l) * (2 * l + 1) + (m1 + l); };
    T.nrot = rot_off(M + 1);
    const int zero = T.nrot;
    std::vector<int> fwd_off{0}, fwd, oz_off{0}, ozt, bwd_off{0}, bwd, sign;
    const int ks = mix ? 1 : -1;  // khi of the -q rotations is ks * khi
    for (int o = 0; o < np; ++o) {
        const int m = g.pm[o], khi = g.pmup[o], mu2 = g.pmu[o] / mrso;
        // forward rotation of output (m, khi, mu2): sum over mup (:505-523)
        for (int mup = -m; mup <= m; ++mup) fwd.push_back(pack_rot_term(pidx(m, mup, mu2), ridx(m, mup, khi), ridx(m, mup, ks * khi)));
        fwd_off.push_back((int)fwd.size());
        // OZ sum of output (m, khi, mu2) (:561-606)
        int ia = ct.ia_start[o];
        for (int n = std::abs(khi); n <= M; ++n)
            for (int nu2 = -n / mrso; nu2 <= n / mrso; ++nu2, ++ia) ozt.push_back(pack_oz_term(ia, pidx(n, khi, std::abs(nu2)), nu2 < 0 ? 1 : 0));
        oz_off.push_back((int)ozt.size());
        // back rotation of output (m, mup, mu2): sum over khi (:626-641)
        for (int k = -m; k <= m; ++k) bwd.push_back(pack_rot_term(pidx(m, k, mu2), ridx(m, khi, k), ridx(m, khi, ks * k)));
        bwd_off.push_back((int)bwd.size());
        sign.push_back(neg1pow(m));
    }
    RotCoef rc;
    build_rot_coef(rc);
    std::vector<int> lvl{0}, rint;
    std::vector<double> rdbl;
    for (int l = 2; l <= M; ++l) {
        const int l1 = l - 1;
        auto U = [&](int m, int m1) { return (std::abs(m) <= l1 && std::abs(m1) <= l1) ? ridx(l1, m, m1) : zero; };
        for (int m = -l; m <= l; ++m) {
            const int m1min = (m > 0) ? 1 : 0;
            for (int m1 = m1min; m1 <= l; ++m1) {
                int x[3] = {ridx(1, 0, 0), ridx(1, 0, 0), ridx(1, 0, 0)}, u[3] = {zero, zero, zero};
                double c[3] = {0, 0, 0};
                if (m1 < l) {
                    if (m == -l) {
                        c[0] = rc.b[l][-m + kRMax][m1 + kRMax]; x[0] = ridx(1, -1, 0); u[0] = U(m + 1, m1);
                    } else if (m == l) {
                        c[0] = rc.b[l][m + kRMax][m1 + kRMax]; x[0] = ridx(1, 1, 0); u[0] = U(m - 1, m1);
                    } else {
                        c[0] = rc.a[l][m + kRMax][m1 + kRMax]; x[0] = ridx(1, 0, 0); u[0] = U(m, m1);
                        c[1] = rc.b[l][m + kRMax][m1 + kRMax]; x[1] = ridx(1, 1, 0); u[1] = U(m - 1, m1);
                        c[2] = rc.b[l][-m + kRMax][m1 + kRMax]; x[2] = ridx(1, -1, 0); u[2] = U(m + 1, m1);
                    }
                } else {
                    if (m == -l) {
                        c[0] = rc.d[l][-m + kRMax]; x[0] = ridx(1, -1, 1); u[0] = U(m + 1, m1 - 1);
                    } else if (m == l) {
                        c[0] = rc.d[l][m + kRMax]; x[0] = ridx(1, 1, 1); u[0] = U(m - 1, m1 - 1);
                    } else {
                        c[0] = rc.c[l][m + kRMax]; x[0] = ridx(1, 0, 1); u[0] = U(m, m1 - 1);
                        c[1] = rc.d[l][m + kRMax]; x[1] = ridx(1, 1, 1); u[1] = U(m - 1, m1 - 1);
                        c[2] = rc.d[l][-m + kRMax]; x[2] = ridx(1, -1, 1); u[2] = U(m + 1, m1 - 1);
                    }
                }
                rint.push_back(ridx(l, m, m1));
                rint.push_back(ridx(l, -m, -m1));
                rint.push_back(neg1pow(m + m1));
                rint.push_back((m == 0 && m1 == 0) ? 1 : 0);
                for (int t = 0; t < 3; ++t) {
                    rint.push_back(x[t]);
                    rint.push_back(u[t]);
                    rdbl.push_back(c[t]);
                }
            }
        }
        lvl.push_back((int)rdbl.size() / kRecDbls);
    }
    T.ints.clear();
    auto put = [&](const std::vector<int> &v) {
        int o = (int)T.ints.size();
        T.ints.insert(T.ints.end(), v.begin(), v.end());
        return o;
    };
    T.fwd_off = put(fwd_off);
    T.fwd_terms = put(fwd);
    T.oz_off = put(oz_off);
    T.oz_terms = put(ozt);
    T.bwd_off = put(bwd_off);
    T.bwd_terms = put(bwd);
    T.sign = put(sign);
    T.lvl_off = put(lvl);
    T.rec_int = put(rint);
    T.dbls = rdbl;
    return true;
}

struct Oz2Args {
    int nx, ny, nz;
    long long N, nk;
    int mmax, np, ncoef, nq;
    double dq, twopi_lx, twopi_ly, twopi_lz;
    int quirks;  // FP64 path: FP32 rounding of the flushed entries and the gamma flush, as the reference
    int n_ints, n_dbls, nrot;
    int fwd_off, fwd_terms, oz_off, oz_terms, bwd_off, bwd_terms, sign, lvl_off, rec_int;
};

template <typename T> __device__ __forceinline__ T round_sp(T x, int q) {  // Fortran default-kind cmplx
    return q ? (T)__double2float_rn((double)x) : x;
}

template <typename C> __device__ __forceinline__ void cfma(C &acc, C a, C b) {  // acc += a*b
    acc.x += a.x * b.x - a.y * b.y;
    acc.y += a.x * b.y + a.y * b.x;
}
template <typename C> __device__ __forceinline__ void cfmac(C &acc, C a, C b) {  // acc += a*conj(b)
    acc.x += a.x * b.x + a.y * b.y;
    acc.y += a.y * b.x - a.x * b.y;
}

// The source species of a multi-species step (Mode 1): their planes, in order.
constexpr int kOzMaxSpecies = 8;
struct OzMix {
    const void *p[kOzMaxSpecies];
    int ns;
};

// per warp: R, ceff and 6 np complex (8 np in Mode 1: the gamma accumulators)
template <typename T>
inline size_t oz2_smem_bytes(const Oz2Args &a, int W, int mode = 0) {
    const size_t per_warp = (size_t)(a.nrot + 1) + a.ncoef + (mode == 1 ? 8 : 6) * a.np;
    return ((a.n_ints * 4 + 15) / 16) * 16 + ((a.n_dbls * sizeof(T) + 15) / 16) * 16 + 32 +
           sizeof(typename Cplx<T>::t) * per_warp * W;
}

// smem: ints | coefficients (T) | flags[2W] | per warp: R[nrot+1], ceff[ncoef], dq, dmq, rq, rmq, gq, gmq
// (Mode 1: and the accumulators aq, amq)
// Mode 0: the single-species step, in place on planes (out and mi unused).  Mode 1: the
// multi-species step (src/module_energy_cproj_mrso_mixture.f90:491-721) for one receiving
// species s2 (c = ctab): gamma_{s2} = sum_s OZ(drho_s) over the source species' planes
// mi.p[s], each source's gamma flushed as the reference does before the sum; R(q) and c are
// formed once per pair and the sum is back-rotated once (the reference back-rotates each
// source's gamma and then sums: the same up to rounding).  Stores gamma_{s2} to out; at
// self-conjugate points it keeps the q result (:685-709); with tables built with mix = true.
template <typename T, int Mode = 0>
__global__ void __launch_bounds__(256) k_oz2(typename Cplx<T>::t *__restrict__ planes,
                                             const typename Cplx<T>::t *__restrict__ ctab, const int *__restrict__ gints,
                                             const double *__restrict__ gdbls, Oz2Args a,
                                             typename Cplx<T>::t *__restrict__ out, OzMix mi) {
    using C = typename Cplx<T>::t;
    extern __shared__ __align__(16) unsigned char oz2_smem[];
    const int W = blockDim.x >> 5;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int *si = reinterpret_cast<int *>(oz2_smem);
    T *sd = reinterpret_cast<T *>(oz2_smem + ((a.n_ints * 4 + 15) / 16) * 16);
    unsigned char *flags = reinterpret_cast<unsigned char *>(sd) + ((a.n_dbls * sizeof(T) + 15) / 16) * 16;
    C *wbase = reinterpret_cast<C *>(flags + 32);
    const int np = a.np;
    const int per_warp = (a.nrot + 1) + a.ncoef + (Mode == 1 ? 8 : 6) * np;
    for (int i = threadIdx.x; i < a.n_ints; i += blockDim.x) si[i] = gints[i];
    for (int i = threadIdx.x; i < a.n_dbls; i += blockDim.x) sd[i] = (T)gdbls[i];
    // persistent: the tables are staged once, then the CTA walks groups of W points
    for (long long k0 = (long long)blockIdx.x * W; k0 < a.nk; k0 += (long long)gridDim.x * W) {
    C *Rw = wbase + (size_t)warp * per_warp;
    C *ceff = Rw + (a.nrot + 1);
    C *dq = ceff + a.ncoef, *dmq = dq + np, *rq = dmq + np, *rmq = rq + np, *gq = rmq + np, *gmq = gq + np;
    C *aq = gmq + np, *amq = aq + np;  // Mode 1 only
    const long long kk = k0 + warp;
    bool active = kk < a.nk;
    int ix = 0, iy = 0, iz = 0, ixm = 0, iym = 0, izm = 0;
    if (active) {
        ix = (int)(kk % a.nx);
        iy = (int)((kk / a.nx) % a.ny);
        iz = (int)(kk / ((long long)a.nx * a.ny));
        ixm = (a.nx - ix) % a.nx;
        iym = (a.ny - iy) % a.ny;
        izm = (a.nz - iz) % a.nz;
        if (iz == 0 || 2 * iz == a.nz)
            if ((long long)iy * a.nx + ix > (long long)iym * a.nx + ixm) active = false;  // partner is the q
    }
    const bool selfconj = active && (ix == ixm && iy == iym && iz == izm);
    const bool nyq = (2 * ix == a.nx) || (2 * iy == a.ny) || (2 * iz == a.nz);
    const int nsrc = Mode == 1 ? mi.ns : 1;
    for (int src = 0; src < nsrc; ++src) {
    __syncthreads();  // tables staged / the previous group's stores (or source's products) have read wbase
    // coalesced load of the W points (side 0) and their partners (side 1)
    const C *pin = Mode == 1 ? static_cast<const C *>(mi.p[src]) : planes;
    for (int e = threadIdx.x; e < 2 * np * W; e += blockDim.x) {
        const int side = e / (np * W), rem = e % (np * W), ip = rem / W, j = rem % W;
        const long long kk = k0 + j;
        if (kk >= a.nk) continue;
        const int ix = (int)(kk % a.nx), iy = (int)((kk / a.nx) % a.ny), iz = (int)(kk / ((long long)a.nx * a.ny));
        long long kidx;
        if (side == 0) kidx = ((long long)iz * a.ny + iy) * a.nx + ix;
        else kidx = ((long long)((a.nz - iz) % a.nz) * a.ny + (a.ny - iy) % a.ny) * a.nx + (a.nx - ix) % a.nx;
        wbase[(size_t)j * per_warp + (a.nrot + 1) + a.ncoef + side * np + ip] = pin[(size_t)ip * a.N + kidx];
    }
    if (src == 0 && lane == 0) {  // after the barrier above: the previous group's stores have read them
        flags[warp] = active ? 1 : 0;
        flags[W + warp] = selfconj ? 1 : 0;
    }
    __syncthreads();
    if (active) {
      if (src == 0) {  // R(q) and c at |q| do not depend on the source species
        const double qx = (ix <= a.nx / 2 ? ix : ix - a.nx) * a.twopi_lx;
        const double qy = (iy <= a.ny / 2 ? iy : iy - a.ny) * a.twopi_ly;
        const double qz = (iz <= a.nz / 2 ? iz : iz - a.nz) * a.twopi_lz;
        // ---- rotation matrix R(q), src/module_rotation.f90:119-247 ----
        if (lane == 0) {
            Rw[0].x = (T)1; Rw[0].y = (T)0;
            Rw[a.nrot].x = (T)0; Rw[a.nrot].y = (T)0;
        }
        if (a.mmax >= 1) {
            T r3[3], r2[3], r1[3];
            if (qx == 0.0 && qy == 0.0 && qz == 0.0) { r3[0] = 0; r3[1] = 0; r3[2] = 1; }
            else { r3[0] = (T)qx; r3[1] = (T)qy; r3[2] = (T)qz; }
            if (r3[0] != (T)0 || r3[1] != (T)0) { r2[0] = -r3[1]; r2[1] = r3[0]; r2[2] = 0; }
            else { r2[0] = 0; r2[1] = r3[2]; r2[2] = -r3[1]; }
            const T n3 = sqrt(r3[0] * r3[0] + r3[1] * r3[1] + r3[2] * r3[2]);
            const T n2 = sqrt(r2[0] * r2[0] + r2[1] * r2[1] + r2[2] * r2[2]);
            for (int i = 0; i < 3; ++i) { r3[i] /= n3; r2[i] /= n2; }
            r1[0] = r2[1] * r3[2] - r2[2] * r3[1];
            r1[1] = r2[2] * r3[0] - r2[0] * r3[2];
            r1[2] = r2[0] * r3[1] - r2[1] * r3[0];
            const T sqrt2 = (T)1.4142135623730950488016887242097;
            if (lane < 9) {
                const int m = lane / 3 - 1, m1 = lane % 3 - 1;
                T f = 0, g = 0;
                if (m == -1 && m1 == -1) { f = (r2[1] + r1[0]) * (T)0.5; g = (r1[1] - r2[0]) * (T)0.5; }
                if (m == -1 && m1 == 0) { f = r3[0] / sqrt2; g = r3[1] / sqrt2; }
                if (m == -1 && m1 == 1) { f = (r2[1] - r1[0]) * (T)0.5; g = (-r1[1] - r2[0]) * (T)0.5; }
                if (m == 0 && m1 == -1) { f = r1[2] / sqrt2; g = -r2[2] / sqrt2; }
                if (m == 0 && m1 == 0) { f = r3[2]; g = 0; }
                if (m == 0 && m1 == 1) { f = -r1[2] / sqrt2; g = -r2[2] / sqrt2; }
                if (m == 1 && m1 == -1) { f = (r2[1] - r1[0]) * (T)0.5; g = (r1[1] + r2[0]) * (T)0.5; }
                if (m == 1 && m1 == 0) { f = -r3[0] / sqrt2; g = r3[1] / sqrt2; }
                if (m == 1 && m1 == 1) { f = (r2[1] + r1[0]) * (T)0.5; g = (r2[0] - r1[1]) * (T)0.5; }
                Rw[1 + lane].x = f;
                Rw[1 + lane].y = g;
            }
            __syncwarp();
            const int *lvl = si + a.lvl_off;
            for (int l = 2; l <= a.mmax; ++l) {
                const int e0 = lvl[l - 2], e1 = lvl[l - 1];
                C val[4];
                int cnt = 0;
                for (int e = e0 + lane; e < e1; e += 32, ++cnt) {
                    const int *ri = si + a.rec_int + kRecInts * e;
                    C s;
                    s.x = 0;
                    s.y = 0;
                    for (int t = 0; t < 3; ++t) {
                        const T cf = sd[kRecDbls * e + t];
                        const C X = Rw[ri[4 + 2 * t]], U = Rw[ri[5 + 2 * t]];
                        // c * (X (x) U), with the reference's grouping
                        s.x += cf * (X.x * U.x - X.y * U.y);
                        s.y += cf * (X.x * U.y + X.y * U.x);
                    }
                    val[cnt] = s;
                }
                __syncwarp();
                cnt = 0;
                for (int e = e0 + lane; e < e1; e += 32, ++cnt) {
                    const int *ri = si + a.rec_int + kRecInts * e;
                    const T sg = (T)ri[2];
                    if (ri[3]) {
                        Rw[ri[0]].x = val[cnt].x;
                        Rw[ri[0]].y = -val[cnt].y;
                    } else {
                        Rw[ri[0]] = val[cnt];
                        Rw[ri[1]].x = sg * val[cnt].x;
                        Rw[ri[1]].y = -sg * val[cnt].y;
                    }
                }
                __syncwarp();
            }
            // flush |Re|, |Im| < epsilon(1.) (:491-492)
            for (int e = lane; e < a.nrot; e += 32) {
                C v = Rw[e];
                if (fabs((double)v.x) < kEpsSp) { v.x = 0; v.y = round_sp(v.y, a.quirks); }
                if (fabs((double)v.y) < kEpsSp) { v.x = round_sp(v.x, a.quirks); v.y = 0; }
                Rw[e] = v;
            }
        }
        // interpolated c (:534-539), staged for the OZ sums
        const double nrm = sqrt(qx * qx + qy * qy + qz * qz);
        const double eff = nrm / a.dq + 1.0;
        const int iq = (int)eff;
        const T alpha = (T)(eff - iq);
        const C *c0 = ctab + (size_t)(iq - 1) * a.ncoef;
        const C *c1 = ctab + (size_t)iq * a.ncoef;
        for (int i = lane; i < a.ncoef; i += 32) {
            const C A = c0[i], B = c1[i];
            C v;
            v.x = alpha * B.x + ((T)1 - alpha) * A.x;
            v.y = alpha * B.y + ((T)1 - alpha) * A.y;
            ceff[i] = v;
        }
        __syncwarp();
      }
        const int *sign = si + a.sign;
        // forward rotation (:505-523)
        {
            const int *off = si + a.fwd_off, *tm = si + a.fwd_terms;
            for (int o = lane; o < np; o += 32) {
                C s, t;
                s.x = s.y = t.x = t.y = 0;
                for (int k = off[o]; k < off[o + 1]; ++k) {
                    const int tt = tm[k], jp = tt & 255, r1i = (tt >> 8) & 2047, r2i = tt >> 19;
                    cfma(s, dq[jp], Rw[r1i]);
                    cfma(t, dmq[jp], Rw[r2i]);
                }
                const T sg = (T)sign[o];
                rq[o] = s;
                t.x *= sg;
                t.y *= sg;
                rmq[o] = t;
            }
        }
        __syncwarp();
        // OZ (:561-606) and the gamma flush (:618-623)
        {
            const int *off = si + a.oz_off, *tm = si + a.oz_terms;
            for (int ip = lane; ip < np; ip += 32) {
                C s, t;
                s.x = s.y = t.x = t.y = 0;
                for (int k = off[ip]; k < off[ip + 1]; ++k) {
                    const int tt = tm[k], ia = tt & 4095, jp = (tt >> 12) & 255, direct = tt >> 20;
                    const C ce = ceff[ia];
                    if (direct) {
                        cfma(s, ce, rq[jp]);
                        cfma(t, ce, rmq[jp]);
                    } else {
                        cfmac(s, ce, rmq[jp]);
                        cfmac(t, ce, rq[jp]);
                    }
                }
                if (a.quirks) {
                    C *vv[2] = {&s, &t};
                    for (int z = 0; z < 2; ++z) {
                        double re = (double)vv[z]->x, im = (double)vv[z]->y;
                        if (fabs(re) < kEpsDp && fabs(im) < kEpsDp) { re = 0.0; im = 0.0; }
                        if (fabs(re) < kEpsDp) { re = 0.0; im = (double)__double2float_rn(im); }
                        if (fabs(im) < kEpsDp) { re = (double)__double2float_rn(re); im = 0.0; }
                        vv[z]->x = (T)re;
                        vv[z]->y = (T)im;
                    }
                }
                gq[ip] = s;
                gmq[ip] = t;
            }
        }
        __syncwarp();
        if (Mode == 1) {  // sum the flushed gamma of every source species
            for (int o = lane; o < np; o += 32) {
                if (src == 0) {
                    aq[o] = gq[o];
                    amq[o] = gmq[o];
                } else {
                    aq[o].x += gq[o].x; aq[o].y += gq[o].y;
                    amq[o].x += gmq[o].x; amq[o].y += gmq[o].y;
                }
            }
            __syncwarp();
        }
    }
    }  // source loop
    if (active) {
        const int *sign = si + a.sign;
        const C *bq = Mode == 1 ? aq : gq, *bmq = Mode == 1 ? amq : gmq;
        // back rotation with conj(R) (:611-641); results replace dq / dmq
        {
            const int *off = si + a.bwd_off, *tm = si + a.bwd_terms;
            for (int o = lane; o < np; o += 32) {
                C s, t;
                s.x = s.y = t.x = t.y = 0;
                for (int k = off[o]; k < off[o + 1]; ++k) {
                    const int tt = tm[k], jp = tt & 255, r1i = (tt >> 8) & 2047, r2i = tt >> 19;
                    cfmac(s, bq[jp], Rw[r1i]);
                    cfmac(t, bmq[jp], Rw[r2i]);
                }
                const T sg = (T)sign[o];
                t.x *= sg;
                t.y *= sg;
                if (selfconj && nyq) t.y = -t.y;
                dq[o] = s;
                dmq[o] = t;
            }
        }
    }
    __syncthreads();
    // coalesced store: q results (not for self-conjugate points) and -q results
    for (int e = threadIdx.x; e < 2 * np * W; e += blockDim.x) {
        const int side = e / (np * W), rem = e % (np * W), ip = rem / W, j = rem % W;
        if (!flags[j]) continue;
        if (flags[W + j] && side == (Mode == 0 ? 0 : 1)) continue;
        const long long kj = k0 + j;
        const int jx = (int)(kj % a.nx), jy = (int)((kj / a.nx) % a.ny), jz = (int)(kj / ((long long)a.nx * a.ny));
        long long kidx;
        if (side == 0) kidx = ((long long)jz * a.ny + jy) * a.nx + jx;
        else kidx = ((long long)((a.nz - jz) % a.nz) * a.ny + (a.ny - jy) % a.ny) * a.nx + (a.nx - jx) % a.nx;
        const C v = wbase[(size_t)j * per_warp + (a.nrot + 1) + a.ncoef + side * np + ip];
        if (Mode == 0) planes[(size_t)ip * a.N + kidx] = v;
        else out[(size_t)ip * a.N + kidx] = v;
    }
    }  // group loop
}

}  // namespace mdft
