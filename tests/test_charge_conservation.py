"""Charge conservation: the discrete Gauss residual stays at round-off.

With cubic cells, the staggered E (Ex at (i+1/2, j, k), Ey at (i, j+1/2, k),
Ez at (i, j, k+1/2)) and the cloud-in-cell charge rho of the particles at the
nodes, the residual

    R = (Ex[i] - Ex[i-1]) + (Ey[j] - Ey[j-1]) + (Ez[k] - Ez[k-1]) - dx * rho

does not change under a step at interior nodes: the Yee curl has zero
discrete divergence, E is updated with -J dx (maxwell.cpp:445-522), and the
12-term segment deposition (deposition.cpp:13-356) satisfies the discrete
continuity equation of linear weighting.  The initial fields are arbitrary,
so R itself is not zero; its change over the steps is compared with the
scale of dx * rho.

Checked for the reference itself (CPU), the FP64 GPU path (round-off of
FP64 atomics) and the mixed GPU path (FP32 round-off).
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.conftest import gpu_available

N = 24
STEPS = 5
KIND = "ref" if O.available("ref", "parity") else "port"


def _state(seed=0):
    dx = 2 * np.pi / 16
    dt = 0.5 * dx
    rng = np.random.default_rng(seed)
    shape = (N, N, N)
    fields = [0.5 * rng.standard_normal(shape) for _ in range(6)]
    m = 3000
    # well inside: a particle moves at most dt/dx = 0.5 cells per step
    x = rng.uniform(6, N - 7, m)
    y = rng.uniform(6, N - 7, m)
    z = rng.uniform(6, N - 7, m)
    u = 0.7 * rng.standard_normal((3, m))
    g = np.sqrt(1 + (u * u).sum(0))
    q = -rng.uniform(0.05, 0.2, m)
    cells = (x.astype(int) * N + y.astype(int)) * N + z.astype(int)
    o = np.argsort(cells, kind="stable")
    parts = {"x": x[o], "y": y[o], "z": z[o], "ux": u[0][o], "uy": u[1][o], "uz": u[2][o], "g": g[o], "q": q[o],
             "cmr": np.full(m, -1.0)}
    return dx, dt, fields, parts


def _rho(p):
    rho = np.zeros((N, N, N))
    i0, j0, k0 = (np.floor(p[a]).astype(int) for a in ("x", "y", "z"))
    fx, fy, fz = p["x"] - i0, p["y"] - j0, p["z"] - k0
    for di, wx in ((0, 1 - fx), (1, fx)):
        for dj, wy in ((0, 1 - fy), (1, fy)):
            for dk, wz in ((0, 1 - fz), (1, fz)):
                np.add.at(rho, (i0 + di, j0 + dj, k0 + dk), p["q"] * wx * wy * wz)
    return rho


def _residual(f12, parts, dx):
    ex, ey, ez = f12[0], f12[1], f12[2]
    div = np.zeros((N, N, N))
    div[1:, :, :] += ex[1:] - ex[:-1]
    div[:, 1:, :] += ey[:, 1:] - ey[:, :-1]
    div[:, :, 1:] += ez[:, :, 1:] - ez[:, :, :-1]
    rho = _rho(parts)
    s = slice(2, N - 2)
    return (div - dx * rho)[s, s, s], np.abs(dx * rho).max()


def _run(region, dx, steps):
    r0, scale = _residual(region.get_fields(), region.get_particles(0) if hasattr(region, "lib")
                          else region.get_particles(), dx)
    region.step(steps)
    p = region.get_particles(0) if hasattr(region, "lib") else region.get_particles()
    r1, _ = _residual(region.get_fields(), p, dx)
    return np.abs(r1 - r0).max() / scale, len(p["x"])


def test_reference_conserves_charge():
    dx, dt, fields, parts = _state()
    r = O.Region(N, N, N, dx, dx, dx, dt, solver=0, pusher=1, kind=KIND)
    r.set_fields(*fields)
    r.init_boundaries()
    r.add_particles(parts)
    err, n = _run(r, dx, STEPS)
    assert n == len(parts["x"])
    assert err < 1e-12, err


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("mixed", 2e-5)])
def test_gpu_conserves_charge(precision, tol):
    if not gpu_available():
        pytest.skip("needs a CUDA device")
    from quill_b200.api import Region
    dx, dt, fields, parts = _state()
    r = Region(N, N, N, dx, dx, dx, dt, precision=precision)
    r.set_fields(*fields)
    r.init_boundaries()
    r.add_particles(0, {k: v for k, v in parts.items() if k != "cmr"})
    err, n = _run(r, dx, STEPS)
    r.close()
    assert n == len(parts["x"])
    assert err < tol, err
