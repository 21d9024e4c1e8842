// Shared pieces of the rotated OZ step (k_oz2.cuh): coefficients of the
// rotation-matrix recursion (src/module_rotation.f90:13-34) and index helpers.
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

}  // namespace mdft
