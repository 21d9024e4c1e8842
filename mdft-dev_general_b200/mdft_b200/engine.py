"""ctypes binding of libmdft_b200.so, mirroring the reference's host calls.

Reference interface (Fortran, dborgis/mdft-dev_general):
  energy_and_gradient(f, df)            src/module_energy_and_gradient.f90:36
  excess_energy(ff, df, print_timers)   src/module_proc_ptrs.f90:3-21
  init_vext                             src/module_vext.f90:14-115
  guess_density                         src/module_density.f90:267-284
  minimization_using_lbfgs              src/energy_minimization.f90:232-290
  pressure_correction                   src/module_pressure_correction.f90:7-156

Arrays use the reference layout xi(no, nx, ny, nz) with io fastest, i.e. numpy
shape (nz, ny, nx, no) in C order.  Errors raise MdftError carrying the
library's message (the reference would `error stop`).  There is no CPU path:
without the compiled library (or without a GPU) construction fails loudly.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PREC_FP64 = 0
PREC_MIXED = 1

_PKG = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def library_path() -> str:
    return os.path.join(_PKG, "libmdft_b200.so")


class MdftError(RuntimeError):
    pass


class _Desc(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("lx", C.c_double), ("ly", C.c_double), ("lz", C.c_double),
                ("mmax", C.c_int), ("mrso", C.c_int), ("temperature", C.c_double), ("n0", C.c_double),
                ("ck_path", C.c_char_p), ("precision", C.c_int), ("device", C.c_int)]


class _Sizes(C.Structure):
    _fields_ = [("ntheta", C.c_int), ("nphi", C.c_int), ("npsi", C.c_int), ("no", C.c_int), ("np", C.c_int),
                ("ncoef", C.c_int), ("nq", C.c_int), ("dv", C.c_double), ("rho0", C.c_double), ("kT", C.c_double),
                ("dq", C.c_double)]


class _MinOpts(C.Structure):
    _fields_ = [("m", C.c_int), ("pgtol", C.c_double), ("ftol_abs", C.c_double), ("itermax", C.c_int),
                ("precision", C.c_int), ("pgtol_mixed", C.c_double), ("polish", C.c_int), ("guni_tol", C.c_double)]


class _MinRes(C.Structure):
    _fields_ = [("f", C.c_double), ("pgnorm", C.c_double), ("iterations", C.c_int), ("evaluations", C.c_int),
                ("status", C.c_int), ("evaluations_mixed", C.c_int), ("guni", C.c_double)]


_DP = C.POINTER(C.c_double)
_FP = C.POINTER(C.c_float)


class _Solute(C.Structure):
    _fields_ = [("nsite", C.c_int), ("q", _DP), ("sig", _DP), ("eps", _DP), ("xyz", _DP), ("handle", C.c_int),
                ("xi_out", _DP)]

# every entry point declared in include/mdft_b200.h: name -> (restype, argtypes)
SIGNATURES = {
    "mdft_create": (C.c_int, [C.POINTER(_Desc), C.POINTER(C.c_void_p)]),
    "mdft_destroy": (C.c_int, [C.c_void_p]),
    "mdft_last_error": (C.c_char_p, []),
    "mdft_get_sizes": (C.c_int, [C.c_void_p, C.POINTER(_Sizes)]),
    "mdft_get_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "mdft_get_weights": (C.c_int, [C.c_void_p, _DP]),
    "mdft_set_vext": (C.c_int, [C.c_void_p, _DP]),
    "mdft_get_vext": (C.c_int, [C.c_void_p, _DP]),
    "mdft_set_constant_correction": (C.c_int, [C.c_void_p, C.c_double]),
    "mdft_energy_and_gradient": (C.c_int, [C.c_void_p, _DP, _DP, _DP, _DP]),
    "mdft_energy_and_gradient_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, _DP, _DP]),
    "mdft_excess_energy": (C.c_int, [C.c_void_p, _DP, _DP, _DP]),
    "mdft_compute_vext": (C.c_int, [C.c_void_p, C.c_int, _DP, _DP, _DP, _DP, C.c_int, _DP, _DP, _DP, _DP,
                                    C.c_double, _DP]),
    "mdft_guess_density": (C.c_int, [C.c_void_p, _DP]),
    "mdft_minimize": (C.c_int, [C.c_void_p, _DP, C.POINTER(_MinOpts), C.POINTER(_MinRes)]),
    "mdft_guess_density_device": (C.c_int, [C.c_void_p, C.c_void_p]),
    "mdft_minimize_device": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(_MinOpts), C.POINTER(_MinRes)]),
    "mdft_get_launch_count": (C.c_int, [C.c_void_p, C.POINTER(C.c_longlong)]),
    "mdft_get_kernel_forms": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), _DP]),
    "mdft_set_wait_failure": (C.c_int, [C.c_void_p, C.c_int]),
    "mdft_ideal_external_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_longlong, C.c_double,
                                              C.c_double, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p]),
    "mdft_pressure_correction": (C.c_int, [C.c_void_p, _DP, C.c_double, C.c_double, _DP]),
    "mdft_pressure_correction_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_double, C.c_double, _DP]),
    "mdft_solve": (C.c_int, [C.c_void_p, C.c_int, _DP, _DP, _DP, _DP, C.c_int, _DP, _DP, _DP, _DP, C.c_double,
                             C.c_double, C.POINTER(_MinOpts), _DP, _DP, C.POINTER(_MinRes)]),
    "mdft_solve_batch": (C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.c_void_p, C.c_int, C.c_int, _DP, _DP, _DP, _DP,
                                   C.c_double, C.c_double, C.POINTER(_MinOpts), _DP, C.c_void_p, C.POINTER(C.c_int)]),
    "mdft_set_timing": (C.c_int, [C.c_void_p, C.c_int]),
    "mdft_get_stage_times": (C.c_int, [C.c_void_p, _DP, C.POINTER(C.c_int)]),
    # density file
    "mdft_write_density_bin": (C.c_int, [C.c_void_p, _DP, C.c_int, _DP, _DP, _DP, _DP, C.POINTER(C.c_int), C.c_int,
                                         C.c_char_p]),
    "mdft_read_density_bin": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int, _DP, _DP, _DP, _DP]),
    # input files
    "mdft_input_read": (C.c_int, [C.c_char_p, C.POINTER(C.c_void_p)]),
    "mdft_input_free": (C.c_int, [C.c_void_p]),
    "mdft_input_nlines": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "mdft_input_line": (C.c_int, [C.c_void_p, C.c_int, C.c_char_p, C.c_int]),
    "mdft_input_get_dp": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int, _DP, C.POINTER(C.c_int)]),
    "mdft_input_get_int": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "mdft_input_get_log": (C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "mdft_input_get_char": (C.c_int, [C.c_void_p, C.c_char_p, C.c_char_p, C.c_int, C.POINTER(C.c_int)]),
    "mdft_desc_from_input": (C.c_int, [C.c_void_p, C.c_char_p, C.c_double, C.c_int, C.c_int, C.POINTER(_Desc)]),
    "mdft_read_solute": (C.c_int, [C.c_char_p, C.c_double, C.c_int, C.POINTER(C.c_int), _DP, _DP, _DP, _DP,
                                   C.POINTER(C.c_int)]),
    "mdft_center_solute": (C.c_int, [C.c_int, _DP, _DP, C.c_int]),
    # learned warm start
    "mdft_warm_net_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "mdft_warm_net_destroy": (C.c_int, [C.c_void_p]),
    "mdft_warm_net_num_params": (C.c_int, [C.c_void_p, C.POINTER(C.c_longlong)]),
    "mdft_warm_net_init": (C.c_int, [C.c_void_p, C.c_ulonglong]),
    "mdft_warm_net_set_params": (C.c_int, [C.c_void_p, _FP, C.c_longlong]),
    "mdft_warm_net_get_params": (C.c_int, [C.c_void_p, _FP, C.c_longlong]),
    "mdft_warm_net_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "mdft_warm_net_forward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "mdft_warm_net_output": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "mdft_warm_net_gradients": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, _FP, _DP]),
    "mdft_warm_net_train_step": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                           C.POINTER(C.c_void_p), C.c_int, C.c_float]),
    "mdft_warm_net_take_loss": (C.c_int, [C.c_void_p, _DP]),
    "mdft_warm_net_launch_count": (C.c_int, [C.c_void_p, C.POINTER(C.c_longlong)]),
    "mdft_warm_net_grid": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "mdft_warm_net_create_n": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "mdft_warm_net_num_outputs": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "mdft_warm_features": (C.c_int, [C.c_void_p, C.c_int, _DP, _DP, _DP, _DP, C.c_int, _DP, _DP, _DP, _DP,
                                     C.c_double, C.c_void_p]),
    "mdft_warm_target": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "mdft_warm_expand": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "mdft_warm_target_n": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "mdft_warm_expand_n": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    "mdft_set_warm_net": (C.c_int, [C.c_void_p, C.c_void_p]),
    "mdft_get_warm_stats": (C.c_int, [C.c_void_p, C.POINTER(C.c_longlong)]),
    # bridge term
    "mdft_set_bridge_cgb": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_double]),
    "mdft_cgb_c00": (C.c_int, [C.c_char_p, C.c_int, _DP]),
    "mdft_bridge_energy": (C.c_int, [C.c_void_p, _DP, _DP, _DP]),
    "mdft_set_bridge_fmt": (C.c_int, [C.c_void_p, C.c_int, C.c_double]),
    "mdft_get_bridge_fmt_params": (C.c_int, [C.c_void_p, _DP]),
    # multi-species solvent
    "mdft_mixture_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int, _DP, C.POINTER(C.c_void_p)]),
    "mdft_mixture_destroy": (C.c_int, [C.c_void_p]),
    "mdft_mixture_energy_and_gradient": (C.c_int, [C.c_void_p, _DP, _DP, _DP, _DP]),
    "mdft_mixture_energy_and_gradient_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, _DP, _DP]),
    "mdft_mixture_minimize": (C.c_int, [C.c_void_p, _DP, C.POINTER(_MinOpts), C.POINTER(_MinRes)]),
}


def lib():
    """Load libmdft_b200.so (raises if it has not been built)."""
    global _LIB
    if _LIB is None:
        path = library_path()
        if not os.path.exists(path):
            raise MdftError("libmdft_b200.so is not built; run __graft_entry__.build() or mdft_b200/build.py")
        L = C.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


def _p(a):
    return None if a is None else a.ctypes.data_as(_DP)


def _check(rc):
    if rc != 0:
        raise MdftError("%s (code %d)" % (lib().mdft_last_error().decode(errors="replace"), rc))


class Engine:
    """One MDFT system on one GPU (grid, solvent, c(k), vext, device buffers)."""

    def __init__(self, n, box, mmax, ck_path, temperature=298.0, n0=0.0333, mrso=2, precision=PREC_FP64, device=0):
        nx, ny, nz = (n, n, n) if np.isscalar(n) else tuple(n)
        lx, ly, lz = (box, box, box) if np.isscalar(box) else tuple(box)
        self._ck = os.fsencode(ck_path)
        d = _Desc(nx, ny, nz, lx, ly, lz, mmax, mrso, temperature, n0, self._ck, precision, device)
        h = C.c_void_p()
        _check(lib().mdft_create(C.byref(d), C.byref(h)))
        self.h = h
        s = _Sizes()
        _check(lib().mdft_get_sizes(self.h, C.byref(s)))
        self.sizes = s
        self.no, self.np = s.no, s.np
        self.dims = (nx, ny, nz)
        self.box = (lx, ly, lz)
        self.shape = (nz, ny, nx, s.no)
        self.dv, self.rho0, self.kT = s.dv, s.rho0, s.kT
        self.device = device
        self.lj_tail = 0.0

    def close(self):
        if getattr(self, "h", None):
            lib().mdft_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- state -------------------------------------------------------------
    @property
    def weights(self):
        w = np.zeros(self.no)
        _check(lib().mdft_get_weights(self.h, _p(w)))
        return w

    @property
    def stream(self) -> int:
        s = C.c_void_p()
        _check(lib().mdft_get_stream(self.h, C.byref(s)))
        return s.value or 0

    def set_vext(self, vext):
        v = np.ascontiguousarray(vext, dtype=np.float64).reshape(self.shape)
        _check(lib().mdft_set_vext(self.h, _p(v)))

    def get_vext(self):
        v = np.empty(self.shape)
        _check(lib().mdft_get_vext(self.h, _p(v)))
        return v

    def set_constant_correction(self, c: float):
        _check(lib().mdft_set_constant_correction(self.h, float(c)))

    # -- the hot path --------------------------------------------------------
    def energy_and_gradient(self, xi, want_grad=True, df_out=None):
        """Return (f, df, terms) with terms = [F_id, F_ext, F_exc, correction]; df = dF/dxi / dv."""
        x = np.ascontiguousarray(xi, dtype=np.float64).reshape(self.shape)
        f = np.zeros(1)
        terms = np.zeros(4)
        df = None
        if want_grad:
            df = df_out if df_out is not None else np.empty(self.shape)
        _check(lib().mdft_energy_and_gradient(self.h, _p(x), _p(f), _p(df), _p(terms)))
        return float(f[0]), df, terms

    def energy_and_gradient_device(self, xi_ptr: int, df_ptr: int | None):
        f = np.zeros(1)
        terms = np.zeros(4)
        _check(lib().mdft_energy_and_gradient_device(self.h, C.c_void_p(xi_ptr), C.c_void_p(df_ptr or 0), _p(f), _p(terms)))
        return float(f[0]), terms

    def excess_energy(self, xi, df=None):
        """Excess term alone; df (if given) is accumulated into, as the reference does."""
        x = np.ascontiguousarray(xi, dtype=np.float64).reshape(self.shape)
        f = np.zeros(1)
        if df is not None:
            assert df.flags.c_contiguous and df.dtype == np.float64 and df.size == x.size
        _check(lib().mdft_excess_energy(self.h, _p(x), _p(f), _p(df)))
        return float(f[0])

    # -- set-up and callers ---------------------------------------------------
    def compute_vext(self, solute, solvent, rvdw=10.0):
        q = np.ascontiguousarray(solute.q, dtype=np.float64)
        sg = np.ascontiguousarray(solute.sig, dtype=np.float64)
        ep = np.ascontiguousarray(solute.eps, dtype=np.float64)
        xyz = np.ascontiguousarray(solute.xyz, dtype=np.float64)
        vq = np.array(solvent.q, dtype=np.float64)
        vs = np.array(solvent.sig, dtype=np.float64)
        ve = np.array(solvent.eps, dtype=np.float64)
        vx = np.array(solvent.xyz, dtype=np.float64)
        lj = np.zeros(1)
        _check(lib().mdft_compute_vext(self.h, len(q), _p(q), _p(sg), _p(ep), _p(xyz), len(vq), _p(vq), _p(vs),
                                       _p(ve), _p(vx), float(rvdw), _p(lj)))
        self.lj_tail = float(lj[0])
        return self.lj_tail

    def set_bridge_cgb(self, version, B6=0.0, sigma=1.0, c00=None, solvent="spce", mmax=None):
        """bridge = "cgb": version 1 'sla', 2 'wda', 0 removes it.  c00 defaults to the
        reference's value for `solvent` at this handle's mmax."""
        if c00 is None and version:
            v = np.zeros(1)
            _check(lib().mdft_cgb_c00(solvent.encode(), int(self.sizes.ntheta - 1 if mmax is None else mmax), _p(v)))
            c00 = float(v[0])
        _check(lib().mdft_set_bridge_cgb(self.h, int(version), float(B6), float(sigma), float(c00 or 0.0)))

    def set_bridge_fmt(self, functional, radius=1.4):
        """bridge = "hard_sphere": functional 1 PY, 2 CS, 0 removes any bridge; radius hs_radius."""
        _check(lib().mdft_set_bridge_fmt(self.h, int(functional), float(radius)))

    def bridge_fmt_params(self):
        """(radius, mu_exc0, Fexc0, nb_k) of the hard-sphere bridge."""
        p = np.zeros(4)
        _check(lib().mdft_get_bridge_fmt_params(self.h, _p(p)))
        return p

    def bridge_energy(self, xi, df=None):
        """energy_bridge(fb, df): returns F_b; adds the bridge gradient to df (in place) when given."""
        x = np.ascontiguousarray(xi, dtype=np.float64).reshape(self.shape)
        fb = np.zeros(1)
        if df is not None and not (df.flags.c_contiguous and df.dtype == np.float64 and df.size == x.size):
            raise MdftError("df must be a contiguous float64 array of xi's size")
        _check(lib().mdft_bridge_energy(self.h, _p(x), _p(fb), _p(df)))
        return float(fb[0])

    def guess_density(self):
        xi = np.empty(self.shape)
        _check(lib().mdft_guess_density(self.h, _p(xi)))
        return xi

    def minimize(self, xi, m=5, pgtol=1e-6, ftol_abs=1e-3, itermax=1000, precision=PREC_FP64, pgtol_mixed=0.0,
                 polish=1, guni_tol=0.0):
        x = np.array(xi, dtype=np.float64, copy=True).reshape(self.shape)
        o = _MinOpts(m, pgtol, ftol_abs, itermax, precision, pgtol_mixed, polish, guni_tol)
        r = _MinRes()
        _check(lib().mdft_minimize(self.h, _p(x), C.byref(o), C.byref(r)))
        return x, dict(f=r.f, pgnorm=r.pgnorm, iterations=r.iterations, evaluations=r.evaluations, status=r.status,
                       evaluations_mixed=r.evaluations_mixed, guni=r.guni)

    def guess_density_device(self, d_xi: int):
        _check(lib().mdft_guess_density_device(self.h, C.c_void_p(d_xi)))

    def minimize_device(self, d_xi: int, m=5, pgtol=1e-6, ftol_abs=1e-3, itermax=1000, precision=PREC_FP64,
                        pgtol_mixed=0.0, polish=1, guni_tol=0.0):
        o = _MinOpts(m, pgtol, ftol_abs, itermax, precision, pgtol_mixed, polish, guni_tol)
        r = _MinRes()
        _check(lib().mdft_minimize_device(self.h, C.c_void_p(d_xi), C.byref(o), C.byref(r)))
        return dict(f=r.f, pgnorm=r.pgnorm, iterations=r.iterations, evaluations=r.evaluations, status=r.status,
                    evaluations_mixed=r.evaluations_mixed, guni=r.guni)

    def set_wait_failure(self, on: bool):
        """Make the gathers report a timed-out wait before issuing any copy (error-path tests)."""
        _check(lib().mdft_set_wait_failure(self.h, 1 if on else 0))

    def kernel_forms(self) -> dict:
        """The FP32 kernel forms in use and the autotuner's stage times (ms, -1: not measured)."""
        f = (C.c_int * 4)()
        ms = np.zeros(6)
        _check(lib().mdft_get_kernel_forms(self.h, f, _p(ms)))
        return dict(project_ring=bool(f[0]), gather_ring=bool(f[1]), oz_factored=bool(f[2]), tuned=bool(f[3]),
                    stage_ms={"project": ms[0:2].tolist(), "oz": ms[2:4].tolist(), "gather": ms[4:6].tolist()})

    @property
    def launch_count(self) -> int:
        c = C.c_longlong()
        _check(lib().mdft_get_launch_count(self.h, C.byref(c)))
        return c.value

    def pressure_correction(self, xi, ftot, lj_tail=None):
        x = np.ascontiguousarray(xi, dtype=np.float64).reshape(self.shape)
        out = np.zeros(4)
        _check(lib().mdft_pressure_correction(self.h, _p(x), float(ftot),
                                              float(self.lj_tail if lj_tail is None else lj_tail), _p(out)))
        return dict(dG=out[0], pmv=out[1], pbulk=out[2], deltaN=out[3])

    def solve(self, solute, solvent, rvdw=10.0, m=5, pgtol=1e-6, ftol_abs=1e-3, itermax=1000, precision=PREC_FP64,
              xi_out=None, pgtol_mixed=0.0, polish=1, guni_tol=0.0):
        """vext -> guess_density -> L-BFGS -> pressure correction for one solute (main.f90's flow)."""
        q = np.ascontiguousarray(solute.q, dtype=np.float64)
        sg = np.ascontiguousarray(solute.sig, dtype=np.float64)
        ep = np.ascontiguousarray(solute.eps, dtype=np.float64)
        xyz = np.ascontiguousarray(solute.xyz, dtype=np.float64)
        vq = np.array(solvent.q, dtype=np.float64)
        vs = np.array(solvent.sig, dtype=np.float64)
        ve = np.array(solvent.eps, dtype=np.float64)
        vx = np.array(solvent.xyz, dtype=np.float64)
        if xi_out is not None:
            assert xi_out.dtype == np.float64 and xi_out.flags.c_contiguous and xi_out.size == int(np.prod(self.shape))
        o = _MinOpts(m, pgtol, ftol_abs, itermax, precision, pgtol_mixed, polish, guni_tol)
        r = _MinRes()
        out = np.zeros(6)
        _check(lib().mdft_solve(self.h, len(q), _p(q), _p(sg), _p(ep), _p(xyz), len(vq), _p(vq), _p(vs), _p(ve), _p(vx),
                                float(rvdw), float(solvent.eps_r), C.byref(o), _p(xi_out), _p(out), C.byref(r)))
        self.lj_tail = float(out[3])
        return dict(dG=out[0], f=out[1], pmv=out[2], lj_tail=out[3], pbulk=out[4], deltaN=out[5], pgnorm=r.pgnorm,
                    iterations=r.iterations, evaluations=r.evaluations, status=r.status,
                    evaluations_mixed=r.evaluations_mixed, guni=r.guni)

    # -- the reference's density file -------------------------------------------
    def write_density_bin(self, path, solute, xi=None, full=False):
        """output/density.bin of the reference for `xi` (None: the last solve's density)."""
        q, sg, ep, xyz = (np.ascontiguousarray(v, dtype=np.float64) for v in (solute.q, solute.sig, solute.eps, solute.xyz))
        Z = None
        if getattr(solute, "Z", None) is not None:
            Z = (C.c_int * len(q))(*[int(z) for z in solute.Z])
        x = None if xi is None else np.ascontiguousarray(xi, dtype=np.float64).reshape(self.shape)
        _check(lib().mdft_write_density_bin(self.h, _p(x), len(q), _p(q), _p(sg), _p(ep), _p(xyz), Z, 1 if full else 0,
                                            str(path).encode()))

    def read_density_bin(self, path, solute, xi_start=None):
        """Restart density from a density.bin onto this grid; points the file does not cover
        keep xi_start's values (default: the bulk guess of the current vext)."""
        sg, ep, xyz = (np.ascontiguousarray(v, dtype=np.float64) for v in (solute.sig, solute.eps, solute.xyz))
        x = np.array(self.guess_density() if xi_start is None else xi_start, dtype=np.float64, copy=True).reshape(self.shape)
        _check(lib().mdft_read_density_bin(self.h, str(path).encode(), len(sg), _p(sg), _p(ep), _p(xyz), _p(x)))
        return x

    # -- learned warm start ---------------------------------------------------
    def warm_features(self, solute, solvent, d_feat: int, rvdw=10.0):
        """The warm-start network's 3 x N input channels for `solute` into device memory."""
        q, sg, ep, xyz = (np.ascontiguousarray(v, dtype=np.float64) for v in (solute.q, solute.sig, solute.eps, solute.xyz))
        vq, vs, ve, vx = (np.array(v, dtype=np.float64) for v in (solvent.q, solvent.sig, solvent.eps, solvent.xyz))
        _check(lib().mdft_warm_features(self.h, len(q), _p(q), _p(sg), _p(ep), _p(xyz), len(vq), _p(vq), _p(vs), _p(ve),
                                        _p(vx), float(rvdw), C.c_void_p(d_feat)))

    def warm_target(self, d_target: int, d_mask: int | None = None, d_xi: int | None = None, nout: int = 4):
        """Training target (nout x N: 4 = the m <= 1 real basis, 2 np = all complex projections as
        real and imaginary planes) and mask (N) from a converged density (default: the last solve)."""
        _check(lib().mdft_warm_target_n(self.h, None if d_xi is None else C.c_void_p(d_xi), int(nout), C.c_void_p(d_target),
                                        None if d_mask is None else C.c_void_p(d_mask)))

    def warm_expand(self, d_pred: int, d_xi: int, nout: int = 4):
        _check(lib().mdft_warm_expand_n(self.h, C.c_void_p(d_pred), int(nout), C.c_void_p(d_xi)))

    def set_warm_net(self, net):
        """Start solves on this engine from `net`'s prediction (None: from the bulk guess)."""
        _check(lib().mdft_set_warm_net(self.h, None if net is None else net.h))
        self._warm = net

    def warm_stats(self):
        s = (C.c_longlong * 2)()
        _check(lib().mdft_get_warm_stats(self.h, s))
        return dict(warm_starts=s[0], fallbacks=s[1])

    def set_timing(self, on=True):
        _check(lib().mdft_set_timing(self.h, 1 if on else 0))

    def stage_times(self):
        ms = np.zeros(5)
        cnt = C.c_int()
        _check(lib().mdft_get_stage_times(self.h, _p(ms), C.byref(cnt)))
        return dict(zip(("project", "fft_forward", "oz", "fft_inverse", "gather"), ms)), cnt.value


class Mixture:
    """A solvent of several species (energy_cproj_mrso_mixture), each an FP64 Engine on one grid.

    Create every species' Engine with n0 = (pure fluid n0) * (its mole fraction), its own
    c(k) file and its vext; the Mixture borrows their buffers and streams, so close it before
    them and do not evaluate on them while it is open.
    """

    def __init__(self, engines, mole_fractions):
        self.engines = list(engines)
        ns = len(self.engines)
        x = np.ascontiguousarray(mole_fractions, dtype=np.float64)
        if x.shape != (ns,):
            raise MdftError("one mole fraction per species")
        hs = (C.c_void_p * ns)(*[e.h for e in self.engines])
        h = C.c_void_p()
        _check(lib().mdft_mixture_create(hs, ns, _p(x), C.byref(h)))
        self.h = h
        self.shape = (ns,) + tuple(self.engines[0].shape)

    def close(self):
        if getattr(self, "h", None):
            lib().mdft_mixture_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def energy_and_gradient(self, xi, want_grad=True):
        """Return (f, df, terms): xi and df of shape (nspec, nz, ny, nx, no), terms as Engine's."""
        x = np.ascontiguousarray(xi, dtype=np.float64).reshape(self.shape)
        f = np.zeros(1)
        terms = np.zeros(4)
        df = np.empty(self.shape) if want_grad else None
        _check(lib().mdft_mixture_energy_and_gradient(self.h, _p(x), _p(f), _p(df), _p(terms)))
        return float(f[0]), df, terms

    def minimize(self, xi, m=5, pgtol=1e-6, ftol_abs=1e-3, itermax=1000, guni_tol=0.0):
        """L-BFGS over every species' xi (FP64); returns (xi, result dict) like Engine.minimize."""
        x = np.array(xi, dtype=np.float64, copy=True).reshape(self.shape)
        o = _MinOpts(m, pgtol, ftol_abs, itermax, PREC_FP64, 0.0, 1, guni_tol)
        r = _MinRes()
        _check(lib().mdft_mixture_minimize(self.h, _p(x), C.byref(o), C.byref(r)))
        return x, dict(f=r.f, pgnorm=r.pgnorm, iterations=r.iterations, evaluations=r.evaluations, status=r.status,
                       guni=r.guni)

    def energy_and_gradient_device(self, xi_ptr: int, df_ptr: int | None):
        f = np.zeros(1)
        terms = np.zeros(4)
        _check(lib().mdft_mixture_energy_and_gradient_device(self.h, C.c_void_p(xi_ptr),
                                                             C.c_void_p(df_ptr) if df_ptr else None, _p(f), _p(terms)))
        return float(f[0]), terms


def solve_batch(engines, solutes, solvent, rvdw=10.0, m=5, pgtol=1e-6, ftol_abs=1e-3, itermax=1000, precision=PREC_FP64,
                pgtol_mixed=0.0, polish=1, handles=None, xi_out=None, guni_tol=0.0):
    """Solve many solutes concurrently: one host worker per engine (each engine has its own
    device buffers and stream), solutes assigned by `handles` (index per solute, -1 or None:
    the next free engine).  xi_out: optional list of host arrays (or None entries) for the
    converged densities.  Returns one result dict per solute, as Engine.solve's."""
    n = len(solutes)
    keep = []
    arr = (_Solute * max(1, n))()
    for i, s in enumerate(solutes):
        q, sg, ep, xyz = (np.ascontiguousarray(v, dtype=np.float64) for v in (s.q, s.sig, s.eps, s.xyz))
        xo = None if xi_out is None else xi_out[i]
        keep += [q, sg, ep, xyz, xo]
        arr[i] = _Solute(len(q), _p(q), _p(sg), _p(ep), _p(xyz), -1 if handles is None else int(handles[i]), _p(xo))
    hs = (C.c_void_p * len(engines))(*[e.h for e in engines])
    vq, vs, ve, vx = (np.array(v, dtype=np.float64) for v in (solvent.q, solvent.sig, solvent.eps, solvent.xyz))
    o = _MinOpts(m, pgtol, ftol_abs, itermax, precision, pgtol_mixed, polish, guni_tol)
    out = np.zeros(6 * max(1, n))
    res = (_MinRes * max(1, n))()
    rc = (C.c_int * max(1, n))()
    _check(lib().mdft_solve_batch(hs, len(engines), C.cast(arr, C.c_void_p), n, len(vq), _p(vq), _p(vs), _p(ve), _p(vx),
                                  float(rvdw), float(solvent.eps_r), C.byref(o), _p(out), C.cast(res, C.c_void_p), rc))
    del keep
    return [dict(dG=out[6 * i], f=out[6 * i + 1], pmv=out[6 * i + 2], lj_tail=out[6 * i + 3], pbulk=out[6 * i + 4],
                 deltaN=out[6 * i + 5], pgnorm=res[i].pgnorm, iterations=res[i].iterations, evaluations=res[i].evaluations,
                 status=res[i].status, evaluations_mixed=res[i].evaluations_mixed, guni=res[i].guni) for i in range(n)]

