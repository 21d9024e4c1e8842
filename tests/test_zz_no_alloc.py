"""The allocation-free entry point mdft_ideal_external_noalloc, for callers that may not
allocate GPU memory (a host whose memory pool owns every device allocation), against the
existing entry points through the C-ABI.  Collected last so that a failure here does not
stop the rest of the suite.

Tolerance as in the other GPU tests: energies 1e-10 relative, gradient 1e-8 of max|df|."""
import ctypes

import numpy as np
import pytest

import cases
from mdft_b200 import Engine, engine

pytestmark = pytest.mark.gpu
SV = cases.SOLVENT


def test_noalloc_matches_existing_entry_points(tmp_path):
    import torch

    c = cases.CASES["mol16_m2"]
    ck = cases.ck_path(tmp_path, c["mmax"])
    e = Engine(c["n"], c["L"], c["mmax"], ck, temperature=SV.temperature, n0=SV.n0)
    e.compute_vext(cases.solute_of(c), SV, rvdw=c["rvdw"])
    vext = e.get_vext()
    xi = cases.xi_of(c, e.shape)
    xi[0, 0, 0, :] = 0.0  # exercise the rho <= eps branch
    f, df_all, terms = e.energy_and_gradient(xi)
    df_exc = np.zeros(e.shape)
    e.excess_energy(xi, df_exc)
    df_id = df_all - df_exc  # the reference's df = (0 + id/ext part) + excess part

    dev = torch.device("cuda", 0)
    t_xi = torch.from_numpy(xi.reshape(-1)).to(dev)
    t_v = torch.from_numpy(vext.reshape(-1)).to(dev)
    t_w = torch.from_numpy(e.weights).to(dev)
    t_df = torch.empty_like(t_xi)
    t_out = torch.zeros(2, dtype=torch.float64, device=dev)
    L = engine.lib()
    npts = int(np.prod(e.shape[:3]))
    scale = np.abs(df_all).max()
    for call in range(2):  # two calls in a row share the library's fixed scratch array
        t_df.fill_(float("nan"))
        t_out.fill_(float("nan"))
        rc = L.mdft_ideal_external_noalloc(t_xi.data_ptr(), t_v.data_ptr(), t_w.data_ptr(), e.no, npts, e.kT, e.rho0,
                                           e.dv, t_df.data_ptr(), t_out.data_ptr(), None)
        assert rc == 0, L.mdft_last_error()
        torch.cuda.synchronize()
        out = t_out.cpu().numpy()
        assert abs(out[0] - terms[0]) <= 1e-10 * abs(f), (call, out, terms)
        assert abs(out[1] - terms[1]) <= 1e-10 * abs(f), (call, out, terms)
        got = t_df.cpu().numpy().reshape(e.shape)
        assert np.abs(got - df_id).max() <= 1e-8 * scale, call
    # sizes beyond the fixed scratch are refused with a message
    rc = L.mdft_ideal_external_noalloc(t_xi.data_ptr(), t_v.data_ptr(), t_w.data_ptr(), e.no, 1 << 21, e.kT, e.rho0,
                                       e.dv, None, t_out.data_ptr(), None)
    assert rc == -1 and b"scratch limit" in L.mdft_last_error()
    e.close()
