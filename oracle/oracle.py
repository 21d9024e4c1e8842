"""ctypes binding of the FP64 CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py as the checker; the product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def build(force: bool = False) -> str:
    so = os.path.join(_HERE, "liboracle.so")
    src = os.path.join(_HERE, "mdft_oracle.c")
    if force or not os.path.exists(so) or os.path.getmtime(so) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE, "liboracle.so"])
    return so


def lib():
    global _LIB
    if _LIB is None:
        _LIB = C.CDLL(build())
        L = _LIB
        dp = C.POINTER(C.c_double)
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                 C.c_int, C.c_int, C.c_double, C.c_double]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_last_error.restype = C.c_char_p
        L.orc_load_ck.argtypes = [C.c_void_p, C.c_char_p]
        L.orc_dims.argtypes = [C.c_void_p, C.POINTER(C.c_int)]
        L.orc_weights.argtypes = [C.c_void_p, dp]
        L.orc_rotm.argtypes = [C.c_void_p, dp]
        L.orc_rho0.argtypes = [C.c_void_p]; L.orc_rho0.restype = C.c_double
        L.orc_dv.argtypes = [C.c_void_p]; L.orc_dv.restype = C.c_double
        L.orc_dq.argtypes = [C.c_void_p]; L.orc_dq.restype = C.c_double
        L.orc_set_vext.argtypes = [C.c_void_p, dp]
        L.orc_get_vext.argtypes = [C.c_void_p, dp]
        L.orc_set_const_corr.argtypes = [C.c_void_p, C.c_double]
        L.orc_ctable.argtypes = [C.c_void_p, dp]
        L.orc_energy_grad.argtypes = [C.c_void_p, dp, dp, dp, dp]
        L.orc_angl2proj.argtypes = [C.c_void_p, dp, dp]
        L.orc_proj2angl.argtypes = [C.c_void_p, dp, dp]
        L.orc_wigner_small_d.restype = C.c_double
        L.orc_wigner_small_d.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double]
        L.orc_gauss_legendre.argtypes = [C.c_int, dp, dp]
        L.orc_rotation_matrix.argtypes = [C.c_int, dp, dp]
        L.orc_charge_corrections.restype = C.c_double
        L.orc_charge_corrections.argtypes = [C.c_double] * 5
        L.orc_qfact.restype = C.c_double
        L.orc_vext.argtypes = [C.c_void_p, C.c_int, dp, dp, dp, dp, C.c_int, dp, dp, dp, dp, C.c_double, dp]
        L.orc_center_solute.argtypes = [C.c_void_p, C.c_int, dp, C.c_int]
        L.orc_guess_density.argtypes = [C.c_void_p, dp]
        L.orc_minimize.argtypes = [C.c_void_p, dp, C.c_int, C.c_double, C.c_double, C.c_int, dp,
                                   C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.orc_set_quirks.argtypes = [C.c_int]
        L.orc_pressure_correction.argtypes = [C.c_void_p, dp, C.c_double, C.c_double, dp]
        L.orc_mixture_energy_grad.argtypes = [C.POINTER(C.c_void_p), C.c_int, dp, dp, dp, dp, dp]
        L.orc_set_bridge_cgb.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_double]
        L.orc_bridge_energy.argtypes = [C.c_void_p, dp, dp, dp]
        L.orc_set_bridge_fmt.argtypes = [C.c_void_p, C.c_int, C.c_double]
        L.orc_mixture_minimize.argtypes = [C.POINTER(C.c_void_p), C.c_int, dp, dp, C.c_int, C.c_double, C.c_double, C.c_int,
                                           dp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.orc_fmt_params.argtypes = [C.c_void_p, dp]
    return _LIB


def _p(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def wigner_small_d(m, mu, mup, theta):
    return lib().orc_wigner_small_d(m, mu, mup, theta)


def gauss_legendre(n):
    x = np.zeros(n); w = np.zeros(n)
    lib().orc_gauss_legendre(n, _p(x), _p(w))
    return x, w


def rotation_matrix(mmax, q):
    W = 2 * mmax + 1
    R = np.zeros((mmax + 1) * W * W * 2)
    lib().orc_rotation_matrix(mmax, _p(np.ascontiguousarray(q, dtype=np.float64)), _p(R))
    return R.view(np.complex128).reshape(mmax + 1, W, W)


def set_quirks(flags: int) -> None:
    """Diagnostics only: 3 (default) keeps both FP32 roundings of the reference."""
    lib().orc_set_quirks(flags)


def qfact():
    return lib().orc_qfact()


def charge_corrections(qnet, L, eps_r, quad_trace, n0):
    return lib().orc_charge_corrections(qnet, L, eps_r, quad_trace, n0)


class Oracle:
    """One MDFT system (grid, solvent, c(k), vext) on the CPU, FP64."""

    def __init__(self, n, box, mmax, ck_path, kT, n0, mrso=2):
        L = lib()
        nx, ny, nz = (n, n, n) if np.isscalar(n) else n
        lx, ly, lz = (box, box, box) if np.isscalar(box) else box
        self.h = L.orc_create(nx, ny, nz, lx, ly, lz, mmax, mrso, kT, n0)
        if not self.h:
            raise RuntimeError(L.orc_last_error().decode())
        if L.orc_load_ck(self.h, ck_path.encode()) != 0:
            raise RuntimeError(L.orc_last_error().decode())
        d = (C.c_int * 7)()
        L.orc_dims(self.h, d)
        self.ntheta, self.nphi, self.npsi, self.no, self.np, self.ncoef, self.nq = list(d)
        self.shape = (nz, ny, nx, self.no)
        self.N = nx * ny * nz
        self.dims = (nx, ny, nz)
        self.box = (lx, ly, lz)

    def close(self):
        if self.h:
            lib().orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def weights(self):
        w = np.zeros(self.no); lib().orc_weights(self.h, _p(w)); return w

    @property
    def rotm(self):
        r = np.zeros(9 * self.no); lib().orc_rotm(self.h, _p(r)); return r.reshape(self.no, 3, 3)

    @property
    def rho0(self):
        return lib().orc_rho0(self.h)

    @property
    def dv(self):
        return lib().orc_dv(self.h)

    @property
    def dq(self):
        return lib().orc_dq(self.h)

    def ctable(self):
        c = np.zeros(self.nq * self.ncoef * 2)
        lib().orc_ctable(self.h, _p(c))
        return c.view(np.complex128).reshape(self.nq, self.ncoef)

    def set_vext(self, v):
        v = np.ascontiguousarray(v, dtype=np.float64).reshape(self.shape)
        lib().orc_set_vext(self.h, _p(v))

    def get_vext(self):
        v = np.zeros(self.shape); lib().orc_get_vext(self.h, _p(v)); return v

    def set_const_corr(self, c):
        lib().orc_set_const_corr(self.h, c)

    def energy_grad(self, xi, want_grad=True):
        xi = np.ascontiguousarray(xi, dtype=np.float64).reshape(self.shape)
        f = np.zeros(1); terms = np.zeros(4)
        df = np.zeros(self.shape) if want_grad else None
        rc = lib().orc_energy_grad(self.h, _p(xi), _p(f), _p(df) if want_grad else None, _p(terms))
        if rc != 0:
            raise RuntimeError(lib().orc_last_error().decode())
        return float(f[0]), df, terms

    def set_bridge_cgb(self, version, B6=0.0, sigma=1.0, c00=-13.665):
        """bridge = "cgb": version 0 none, 1 'sla', 2 'wda'; c00 the solvent's c(k=0)."""
        if lib().orc_set_bridge_cgb(self.h, version, B6, sigma, c00) != 0:
            raise RuntimeError(lib().orc_last_error().decode())

    def set_bridge_fmt(self, functional, radius=1.4):
        """bridge = "hard_sphere": functional 1 PY, 2 CS, 0 removes it; radius hs_radius."""
        if lib().orc_set_bridge_fmt(self.h, functional, radius) != 0:
            raise RuntimeError(lib().orc_last_error().decode())

    def fmt_params(self):
        """(radius, excess chemical potential, bulk grand potential Fexc0, nb_k)."""
        p = np.zeros(4); lib().orc_fmt_params(self.h, _p(p)); return p

    def bridge_energy(self, xi, df=None):
        """energy_bridge(fb, df): returns fb; adds the bridge gradient to df when given."""
        xi = np.ascontiguousarray(xi, dtype=np.float64).reshape(self.shape)
        fb = np.zeros(1)
        if df is not None:
            assert df.flags.c_contiguous and df.dtype == np.float64
        if lib().orc_bridge_energy(self.h, _p(xi), _p(fb), _p(df) if df is not None else None) != 0:
            raise RuntimeError(lib().orc_last_error().decode())
        return float(fb[0])

    def angl2proj(self, o):
        o = np.ascontiguousarray(o, dtype=np.float64)
        p = np.zeros(2 * self.np); lib().orc_angl2proj(self.h, _p(o), _p(p)); return p.view(np.complex128)

    def proj2angl(self, p):
        p = np.ascontiguousarray(p, dtype=np.complex128).view(np.float64)
        o = np.zeros(self.no); lib().orc_proj2angl(self.h, _p(p), _p(o)); return o

    def center_solute(self, xyz, translate=True):
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).copy()
        lib().orc_center_solute(self.h, len(xyz), _p(xyz), 1 if translate else 0)
        return xyz

    def compute_vext(self, solute, solvent, rvdw=10.0):
        s = solute
        q = np.ascontiguousarray(s.q, dtype=np.float64); sg = np.ascontiguousarray(s.sig, dtype=np.float64)
        ep = np.ascontiguousarray(s.eps, dtype=np.float64); xyz = np.ascontiguousarray(s.xyz, dtype=np.float64)
        vq = np.array(solvent.q, dtype=np.float64); vs = np.array(solvent.sig, dtype=np.float64)
        ve = np.array(solvent.eps, dtype=np.float64); vx = np.array(solvent.xyz, dtype=np.float64)
        lj = np.zeros(1)
        rc = lib().orc_vext(self.h, len(q), _p(q), _p(sg), _p(ep), _p(xyz), len(vq), _p(vq), _p(vs), _p(ve), _p(vx),
                            rvdw, _p(lj))
        if rc != 0:
            raise RuntimeError(lib().orc_last_error().decode())
        return float(lj[0])

    def guess_density(self):
        xi = np.zeros(self.shape); lib().orc_guess_density(self.h, _p(xi)); return xi

    def minimize(self, xi, m=5, pgtol=1e-6, tol=1e-3, itermax=1000):
        xi = np.ascontiguousarray(xi, dtype=np.float64).reshape(self.shape).copy()
        f = np.zeros(1); nfg = C.c_int(); it = C.c_int(); st = C.c_int()
        rc = lib().orc_minimize(self.h, _p(xi), m, pgtol, tol, itermax, _p(f), C.byref(nfg), C.byref(it), C.byref(st))
        if rc != 0:
            raise RuntimeError(lib().orc_last_error().decode())
        return xi, float(f[0]), nfg.value, it.value, st.value

    def pressure_correction(self, xi, ftot, lj_corr):
        out = np.zeros(4)
        rc = lib().orc_pressure_correction(self.h, _p(np.ascontiguousarray(xi, dtype=np.float64)), ftot, lj_corr, _p(out))
        if rc != 0:
            raise RuntimeError(lib().orc_last_error().decode())
        return dict(dG=out[0], pmv=out[1], pbulk=out[2], deltaN=out[3])


def mixture_energy_grad(species, mole_fractions, xi, want_grad=True):
    """energy_and_gradient of a multi-species solvent (energy_cproj_mrso_mixture).

    species: Oracle objects on one grid, each created with its n0 times its mole fraction,
    with its own c(k) table and vext; xi: (nspec, *shape).  Returns (F, df, terms) with
    df of xi's shape and terms {F_id, F_ext, F_exc, corrections}.
    """
    ns = len(species)
    shape = (ns,) + tuple(species[0].shape)
    xi = np.ascontiguousarray(xi, dtype=np.float64).reshape(shape)
    x = np.ascontiguousarray(mole_fractions, dtype=np.float64)
    hs = (C.c_void_p * ns)(*[o.h for o in species])
    f = np.zeros(1); terms = np.zeros(4)
    df = np.zeros(shape) if want_grad else None
    rc = lib().orc_mixture_energy_grad(hs, ns, _p(x), _p(xi), _p(f), _p(df) if want_grad else None, _p(terms))
    if rc != 0:
        raise RuntimeError(lib().orc_last_error().decode())
    return float(f[0]), df, terms


def mixture_minimize(species, mole_fractions, xi, m=5, pgtol=1e-6, tol=1e-3, itermax=1000):
    """L-BFGS over every species' xi at once; returns (xi, f, evaluations, iterations, status)."""
    ns = len(species)
    shape = (ns,) + tuple(species[0].shape)
    x = np.ascontiguousarray(xi, dtype=np.float64).reshape(shape).copy()
    fr = np.ascontiguousarray(mole_fractions, dtype=np.float64)
    hs = (C.c_void_p * ns)(*[o.h for o in species])
    f = np.zeros(1); nfg = C.c_int(); it = C.c_int(); st = C.c_int()
    rc = lib().orc_mixture_minimize(hs, ns, _p(fr), _p(x), m, pgtol, tol, itermax, _p(f), C.byref(nfg), C.byref(it),
                                    C.byref(st))
    if rc != 0:
        raise RuntimeError(lib().orc_last_error().decode())
    return x, float(f[0]), nfg.value, it.value, st.value
