"""The reference's input files through the library's readers (include/mdft_b200.h).

  dft.in     getinput%dp/int/log/char (src/module_input.f90), the grid and thermo tags
             of init_grid / init_thermo (src/module_grid.f90:62-95, src/module_thermo.f90:25)
  solute.in  read_solute (src/module_solute.f90:36-52) and mv_solute_to_center (:146-187)

    from mdft_b200 import inputs
    d = inputs.DftInput("dft.in")
    e = d.engine("ck.txt")                        # Engine on dft.in's grid, mmax, temperature
    sol = inputs.read_solute("solute.in", d.dp("solute_charges_scale_factor", 1.0))
    sol.xyz = inputs.center_solute(sol.xyz, e.box, d.log("translate_solute_to_center", True))
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import engine as E
from . import synth


class DftInput:
    """A dft.in file after the reference's line clean-up; tag getters with defaults."""

    def __init__(self, path: str):
        h = C.c_void_p()
        E._check(E.lib().mdft_input_read(str(path).encode(), C.byref(h)))
        self.h = h.value

    def close(self):
        if getattr(self, "h", None):
            E.lib().mdft_input_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def lines(self) -> list[str]:
        n = C.c_int()
        E._check(E.lib().mdft_input_nlines(self.h, C.byref(n)))
        buf = C.create_string_buffer(128)
        out = []
        for i in range(n.value):
            E._check(E.lib().mdft_input_line(self.h, i, buf, 128))
            out.append(buf.value.decode())
        return out

    def _get(self, fn, ctype, tag, default, n):
        vals = (ctype * n)(*(([default] * n) if np.isscalar(default) or default is None else default)) \
            if default is not None else (ctype * n)()
        found = C.c_int()
        E._check(fn(self.h, tag.encode(), n, vals, C.byref(found)))
        if not found.value and default is None:
            raise E.MdftError("tag %s not found in dft.in and no default" % tag)
        return vals[0] if n == 1 else tuple(vals)

    def dp(self, tag: str, default=None, n: int = 1):
        return self._get(E.lib().mdft_input_get_dp, C.c_double, tag, default, n)

    def int(self, tag: str, default=None, n: int = 1):
        return self._get(E.lib().mdft_input_get_int, C.c_int, tag, default, n)

    def log(self, tag: str, default=None) -> bool:
        v = C.c_int(1 if default else 0)
        found = C.c_int()
        E._check(E.lib().mdft_input_get_log(self.h, tag.encode(), C.byref(v), C.byref(found)))
        if not found.value and default is None:
            raise E.MdftError("tag %s not found in dft.in and no default" % tag)
        return bool(v.value)

    def char(self, tag: str, default=None) -> str:
        buf = C.create_string_buffer(64)
        found = C.c_int()
        E._check(E.lib().mdft_input_get_char(self.h, tag.encode(), buf, 64, C.byref(found)))
        if not found.value:
            if default is None:
                raise E.MdftError("tag %s not found in dft.in and no default" % tag)
            return default
        return buf.value.decode()

    def desc(self, ck_path: str, n0: float = 0.0333, precision: int = E.PREC_FP64, device: int = 0) -> dict:
        """Engine arguments of the grid and thermo this dft.in describes."""
        ck = str(ck_path).encode()
        d = E._Desc()
        E._check(E.lib().mdft_desc_from_input(self.h, ck, float(n0), precision, device, C.byref(d)))
        return dict(n=(d.nx, d.ny, d.nz), box=(d.lx, d.ly, d.lz), mmax=d.mmax, mrso=d.mrso, temperature=d.temperature,
                    n0=d.n0, ck_path=ck_path, precision=d.precision, device=d.device)

    def engine(self, ck_path: str, n0: float = 0.0333, precision: int = E.PREC_FP64, device: int = 0) -> E.Engine:
        a = self.desc(ck_path, n0, precision, device)
        return E.Engine(a["n"], a["box"], a["mmax"], a["ck_path"], temperature=a["temperature"], n0=a["n0"],
                        mrso=a["mrso"], precision=a["precision"], device=a["device"])


def read_solute(path: str, charge_scale: float = 1.0) -> synth.Solute:
    n = C.c_int()
    E._check(E.lib().mdft_read_solute(str(path).encode(), float(charge_scale), 0, C.byref(n), None, None, None, None, None))
    k = n.value
    q, sg, ep = np.zeros(k), np.zeros(k), np.zeros(k)
    xyz = np.zeros((k, 3))
    Z = (C.c_int * max(1, k))()
    E._check(E.lib().mdft_read_solute(str(path).encode(), float(charge_scale), k, C.byref(n), E._p(q), E._p(sg), E._p(ep),
                                      E._p(xyz), Z))
    return synth.Solute(q=q, sig=sg, eps=ep, xyz=xyz, Z=np.array(Z[:k], dtype=int))


def center_solute(xyz, box, translate: bool = True) -> np.ndarray:
    out = np.array(xyz, dtype=np.float64, copy=True).reshape(-1, 3)
    b = np.ascontiguousarray(box if not np.isscalar(box) else (box,) * 3, dtype=np.float64)
    E._check(E.lib().mdft_center_solute(len(out), E._p(out), E._p(b), 1 if translate else 0))
    return out
