"""CPU oracle of the learned warm start (TEST INFRASTRUCTURE ONLY: imported by tests/ and
__graft_entry__.smoke() as the checker, never by the product).

* The network in torch float64 on the CPU -- periodic 3x3x3 convolutions
  (circular padding), 2x2x2 stride-2 convolutions and their transposes, GELU (erf form),
  skip additions, a pointwise head -- with the library's flat parameter order, so that
  autograd gives the reference gradients of the library's forward and backward kernels.
* numpy restatements of the solver-side kernels: the input channels from the solute
  sites, the m <= 1 log-density projections of a density with their loss mask, and the
  starting density built from projections; the same for the projection form (all np
  complex projections of the log-density by the C oracle's angl2proj, the start by its
  proj2angl).

The warm start has no counterpart in the reference (whose solves start from
guess_density, src/module_density.f90:267-284); the definitions restated here are the
library's own (csrc/warmnet.cu, csrc/warmstart.cuh).
"""
from __future__ import annotations

import math

import numpy as np

# (kind, input tensor, output tensor, cin, cout, skip tensor, GELU); the head's cout is the
# network's output count (4 here; layers(nout) for other widths)
CONV3, DOWN, UP, HEAD = 0, 1, 2, 3
LAYERS = [
    (CONV3, 0, 1, 3, 16, -1, 1), (CONV3, 1, 2, 16, 16, -1, 1), (DOWN, 2, 3, 16, 32, -1, 1),
    (CONV3, 3, 4, 32, 32, -1, 1), (DOWN, 4, 5, 32, 64, -1, 1), (CONV3, 5, 6, 64, 64, -1, 1),
    (DOWN, 6, 7, 64, 128, -1, 1), (CONV3, 7, 8, 128, 128, -1, 1), (UP, 8, 9, 128, 64, 6, 0),
    (CONV3, 9, 10, 64, 64, -1, 1), (UP, 10, 11, 64, 32, 4, 0), (CONV3, 11, 12, 32, 32, -1, 1),
    (UP, 12, 13, 32, 16, 2, 0), (CONV3, 13, 14, 16, 16, -1, 1), (HEAD, 14, 15, 16, 4, -1, 0),
]


def weight_shape(kind, cin, cout):
    if kind == CONV3:
        return (cout, cin, 3, 3, 3)
    if kind == DOWN:
        return (cout, cin, 2, 2, 2)
    if kind == UP:
        return (cin, cout, 2, 2, 2)
    return (cout, cin, 1, 1, 1)


def layers(nout: int = 4):
    return [(k, x, y, ci, nout if k == HEAD else co, sk, g) for k, x, y, ci, co, sk, g in LAYERS]


def num_params(nout: int = 4) -> int:
    return sum(int(np.prod(weight_shape(k, ci, co))) + co for k, _, _, ci, co, _, _ in layers(nout))


def unpack(flat, torch, nout: int = 4):
    """Flat parameter vector (per layer: weights, then biases) -> list of (W, b) tensors."""
    out, off = [], 0
    for k, _, _, ci, co, _, _ in layers(nout):
        shp = weight_shape(k, ci, co)
        n = int(np.prod(shp))
        out.append((flat[off:off + n].reshape(shp), flat[off + n:off + n + co]))
        off += n + co
    assert off == flat.shape[0]
    return out


def forward(flat, x, torch, nout: int = 4):
    """x: (3, nz, ny, nx) float64 tensor; flat: parameter tensor (the library uses BF16
    weights, so pass weights rounded to BF16 for a like-for-like comparison)."""
    F = torch.nn.functional
    params = unpack(flat, torch, nout)
    t = {0: x.unsqueeze(0)}
    for (k, xi, yi, ci, co, skip, gelu), (W, b) in zip(layers(nout), params):
        a = t[xi]
        if k == CONV3:
            y = F.conv3d(F.pad(a, (1, 1, 1, 1, 1, 1), mode="circular"), W, b)
        elif k == DOWN:
            y = F.conv3d(a, W, b, stride=2)
        elif k == UP:
            y = F.conv_transpose3d(a, W, b, stride=2) + t[skip]
        else:
            y = F.conv3d(a, W, b)
        t[yi] = F.gelu(y) if gelu else y
    return t[15][0]


def loss(y, target, mask):
    """sum_v mask_v sum_c (y - t)^2 / (C N), the library's training loss (C outputs)."""
    n = y.shape[1] * y.shape[2] * y.shape[3]
    return (((y - target) ** 2).sum(0) * mask).sum() / (float(y.shape[0]) * n)


def bf16_round(x: np.ndarray) -> np.ndarray:
    b = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32)


def bf16_weights(flat: np.ndarray, nout: int = 4) -> np.ndarray:
    """The library's kernel parameters: weights rounded to BF16, biases kept FP32."""
    out = np.array(flat, dtype=np.float32, copy=True)
    off = 0
    for k, _, _, ci, co, _, _ in layers(nout):
        n = int(np.prod(weight_shape(k, ci, co)))
        out[off:off + n] = bf16_round(out[off:off + n])
        off += n + co
    return out


# ---------------------------------------------------------------------------
# solver-side kernels
QFACT = (1.602176565e-19 ** 2 * 1.0e-3 * 6.02214129e23 / (4.0 * math.pi * 8.854187817e-12 * 1.0e-10))
SMEAR = 0.5
FLOOR, CEIL = -8.0, 4.0   # clamp of the target's ln(rho/rho0)
START_FLOOR = -2.0        # clamp of the start's ln(rho/rho0)


def features(dims, box, solute, solvent, kT, rvdw):
    """3 x (nz, ny, nx) channels: asinh(min(v_LJ/kT, 1e4))/4, asinh(V/kT)/4, site density."""
    from scipy.special import erf
    nx, ny, nz = dims
    lx, ly, lz = box
    iz, iy, ix = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    r = np.stack([ix * (lx / nx), iy * (ly / ny), iz * (lz / nz)], -1)
    L = np.array([lx, ly, lz])
    sig_s = eps_s = 0.0
    for s, e in zip(solvent.sig, solvent.eps):
        if e > 0:
            sig_s, eps_s = s, e
            break
    vlj = np.zeros((nz, ny, nx))
    vq = np.zeros((nz, ny, nx))
    dens = np.zeros((nz, ny, nx))
    for k in range(len(solute.q)):
        d = r - np.asarray(solute.xyz[k])
        d -= L * np.rint(d / L)
        r2 = (d * d).sum(-1)
        if solute.eps[k] > 0 and eps_s > 0:
            sg = 0.5 * (solute.sig[k] + sig_s)
            e = math.sqrt(solute.eps[k] * eps_s)
            with np.errstate(divide="ignore", over="ignore", invalid="ignore"):
                s6 = (sg * sg / r2) ** 3
                v = np.where(r2 < 1e-6, 1e10, 4 * e * (s6 * s6 - s6))
            vlj += np.where(r2 <= rvdw * rvdw, v, 0.0)
        if solute.q[k] != 0:
            rr = np.sqrt(r2)
            with np.errstate(divide="ignore", invalid="ignore"):
                v = np.where(rr < 1e-6, solute.q[k] * math.sqrt(2 / math.pi) / SMEAR,
                             solute.q[k] * erf(rr / (math.sqrt(2) * SMEAR)) / rr)
            vq += v
        dens += np.exp(-r2 / (2 * SMEAR * SMEAR))
    vq *= QFACT
    return np.stack([0.25 * np.arcsinh(np.minimum(vlj / kT, 1e4)), 0.25 * np.arcsinh(vq / kT), dens])


def orientation_table(rotm, w):
    """(no, 4): the molecular z axis R(omega) z in the lab frame, and the weight."""
    R = np.asarray(rotm).reshape(-1, 3, 3)
    return np.concatenate([R[:, :, 2], np.asarray(w)[:, None]], 1)


def target(xi, vext, table, vmax):
    """xi, vext: (nz, ny, nx, no).  Returns the 4 projections of clamp(2 ln xi) and the mask."""
    with np.errstate(divide="ignore"):
        f = np.where(xi > 0, 2.0 * np.log(np.where(xi > 0, xi, 1.0)), FLOOR)
    f = np.clip(f, FLOOR, CEIL)
    u, w = table[:, :3], table[:, 3]
    a0 = (f * w).sum(-1) / w.sum()
    ak = [(f * w * u[:, k]).sum(-1) / (w * u[:, k] ** 2).sum() for k in range(3)]
    mask = (vext < vmax).any(-1).astype(np.float64)
    return np.stack([a0] + ak), mask


def expand(pred, vext, table, vmax):
    """pred: 4 x (nz, ny, nx) -> xi (nz, ny, nx, no)."""
    u = table[:, :3]
    f = pred[0][..., None] + sum(pred[k + 1][..., None] * u[:, k] for k in range(3))
    f = np.clip(f, START_FLOOR, CEIL)
    return np.where(vext >= vmax, 0.0, np.exp(0.5 * f))


# projection form -----------------------------------------------------------
def angular_maps(orc):
    """(A, B) of the C oracle: A (no, np) complex with angl2proj(o) = o @ A; B (2 np, no) real
    with proj2angl(p) = sum_k [Re p, Im p]_k B_k (both maps are linear)."""
    no, np_ = orc.no, orc.np
    A = np.stack([orc.angl2proj(np.eye(no)[i]) for i in range(no)])
    B = np.zeros((2 * np_, no))
    for ip in range(np_):
        for c, val in ((0, 1.0), (1, 1.0j)):
            p = np.zeros(np_, dtype=np.complex128)
            p[ip] = val
            B[2 * ip + c] = orc.proj2angl(p)
    return A, B


def target_proj(xi, vext, A, vmax):
    """xi, vext: (nz, ny, nx, no).  Returns the 2 np planes (Re, Im of each projection, in
    the projection order) of clamp(2 ln xi), and the mask."""
    with np.errstate(divide="ignore"):
        f = np.where(xi > 0, 2.0 * np.log(np.where(xi > 0, xi, 1.0)), FLOOR)
    f = np.clip(f, FLOOR, CEIL)
    p = f @ A  # (nz, ny, nx, np) complex
    planes = np.stack([p.real, p.imag], axis=-1).reshape(p.shape[:3] + (-1,))
    mask = (vext < vmax).any(-1).astype(np.float64)
    return np.moveaxis(planes, -1, 0), mask


def expand_proj(pred, vext, B, vmax):
    """pred: 2 np x (nz, ny, nx) -> xi (nz, ny, nx, no)."""
    f = np.tensordot(np.moveaxis(pred, 0, -1), B, axes=([3], [0]))
    f = np.clip(f, START_FLOOR, CEIL)
    return np.where(vext >= vmax, 0.0, np.exp(0.5 * f))
