"""Hand-written discrete adjoint (qp_adjoint_energy) and its torch binding.

The adjoint has no reference counterpart; it is checked against central
finite differences of the library's own FP64 forward, h = 1e-6 relative to
the scale of each perturbed quantity.  Tolerance: 1e-4 relative to the
finite difference, plus 1e-7 of the largest gradient component for entries
whose gradient is near zero (finite-difference noise is about 1e-10 of the
loss here).
"""
import math

import numpy as np
import pytest
import torch

from quill_b200.adjoint import FinalElectronEnergy, SlabLaserCase, SlabLaserProblem, hermite_functions
from tests.conftest import gpu_available

H_REL = 1e-6
RTOL = 1e-4
ATOL_OF_MAX = 1e-7


def _small_case(**kw) -> SlabLaserCase:
    """No particle reaches a boundary within the steps, so that the loss is
    a smooth function of every input (an erased particle makes it jump)."""
    base = dict(nx=48, ny=28, nz=28, nsteps=24, every=5, ppc=2, height=0.5, centre=24.0, width=6.0, edge=1.5,
                margin=2.0, transverse_gap=9, a0=0.5, fwhm_lambda=0.7, waist_lambda=0.5, n_modes=8, seed=3)
    base.update(kw)
    return SlabLaserCase(**base)


def _close(g_adj, g_fd, gmax):
    return abs(g_adj - g_fd) <= RTOL * abs(g_fd) + ATOL_OF_MAX * gmax


# ---------------------------------------------------------------- CPU ----

def test_hermite_functions_orthonormal():
    u = torch.linspace(-12, 12, 24001, dtype=torch.float64)
    h = hermite_functions(u, 8)
    w = torch.exp(-u * u) * (u[1] - u[0])
    gram = (h[:, None, :] * h[None, :, :] * w).sum(-1) / math.sqrt(math.pi)
    assert torch.allclose(gram, torch.eye(8, dtype=torch.float64), atol=1e-10)


def test_slab_weights_and_laser_fields_shapes():
    p = SlabLaserProblem(_small_case())
    coef, slab = p.nominal()
    q = p.weights(slab)
    assert q.shape == (p.n_particles,)
    x = p.particles["x"]
    want = -0.25 * (np.tanh((x - 24.0 + 3.0) / 1.5) - np.tanh((x - 24.0 - 3.0) / 1.5)) / 2
    assert np.allclose(q.numpy(), want, rtol=1e-14, atol=0)
    assert (q < 0).all() and q.min() < -0.2
    f = p.fields(coef)
    assert f.shape == (6, 48, 28, 28) and f.dtype == torch.float64
    assert f[[0, 2, 3, 4]].abs().max() == 0
    assert f[1].abs().max() > 0.3
    # the fundamental mode alone is the Gaussian profile
    j, k = 11, 15
    yv, zv = j + 0.5 - 14, k - 14
    g = math.exp(-(yv * yv + zv * zv) / p.w ** 2)
    i = int(round(p.xc))
    a = (i - p.xc) / p.xs
    want = 0.5 * math.cos(0.5 * math.pi * a) ** 2 * g * math.cos((i - p.xc) * p.case.dx)
    assert abs(f[1, i, j, k].item() - want) < 1e-12


def test_parameter_gradients_reach_the_leaves_through_the_maps():
    """dL/dfields and dL/dq from the adjoint are chained by autograd: with a
    stand-in adjoint (L = <a, fields> + <b, q>) the leaves' gradients equal
    the chain rule computed by hand."""
    p = SlabLaserProblem(_small_case())
    coef, slab = p.nominal()
    coef.requires_grad_(True)
    slab.requires_grad_(True)
    gen = torch.Generator().manual_seed(1)
    a = torch.randn(6, 48, 28, 28, dtype=torch.float64, generator=gen)
    b = torch.randn(p.n_particles, dtype=torch.float64, generator=gen)

    class Stand(torch.autograd.Function):
        @staticmethod
        def forward(ctx, f, q):
            return (a * f).sum() + (b * q).sum()

        @staticmethod
        def backward(ctx, g):
            return g * a, g * b

    Stand.apply(p.fields(coef), p.weights(slab)).backward()
    c2 = coef.detach().clone().requires_grad_(True)
    s2 = slab.detach().clone().requires_grad_(True)
    ((a * p.fields(c2)).sum() + (b * p.weights(s2)).sum()).backward()
    assert torch.allclose(coef.grad, c2.grad) and torch.allclose(slab.grad, s2.grad)


# ---------------------------------------------------------------- GPU ----

gpu = pytest.mark.gpu


def _require_gpu():
    if not gpu_available():
        pytest.skip("needs a CUDA device")


def _random_fields(p, seed=0, scale=0.1):
    coef, _ = p.nominal()
    f = p.fields(coef).numpy().copy()
    rng = np.random.default_rng(seed)
    # smooth extra fields in every component
    nx, ny, nz = f.shape[1:]
    i = np.arange(nx)[:, None, None]
    j = np.arange(ny)[None, :, None]
    k = np.arange(nz)[None, None, :]
    for c in range(6):
        a, b, d = rng.uniform(0.1, 0.5, 3)
        ph = rng.uniform(0, 2 * np.pi, 3)
        f[c] += scale * np.sin(a * i + ph[0]) * np.cos(b * j + ph[1]) * np.sin(d * k + ph[2])
    return f


@gpu
def test_adjoint_leaves_state_and_matches_forward_loss():
    _require_gpu()
    p = SlabLaserProblem(_small_case())
    coef, slab = p.nominal()
    f = _random_fields(p)
    q = p.weights(slab).numpy()
    r = p.setup.region(f, q)
    f0 = r.get_fields()
    p0 = r.get_particles(0)
    loss, gf, gq = r.adjoint_energy(p.setup.nsteps, p.setup.every)
    f1 = r.get_fields()
    p1 = r.get_particles(0)
    assert np.array_equal(f0, f1)
    for key in ("x", "y", "z", "ux", "uy", "uz", "g", "q", "cell"):
        assert np.array_equal(p0[key], p1[key]), key
    fwd = r.step(p.setup.nsteps)[-1].energy_e
    assert r.count(0) == p.n_particles  # nothing erased: the loss is smooth in the inputs
    r.close()
    assert loss > 0 and abs(loss - fwd) <= 1e-12 * abs(fwd)
    assert gf.shape == (6, 48, 28, 28) and gq.shape == (p.n_particles,)
    assert np.isfinite(gf).all() and np.isfinite(gq).all()


@gpu
def test_adjoint_independent_of_checkpoint_interval():
    _require_gpu()
    p = SlabLaserProblem(_small_case())
    _, slab = p.nominal()
    f = _random_fields(p)
    q = p.weights(slab).numpy()
    out = []
    for every in (1, 5, 24, 100):
        r = p.setup.region(f, q)
        out.append(r.adjoint_energy(p.setup.nsteps, every))
        r.close()
    l0, gf0, gq0 = out[0]
    for l1, gf1, gq1 in out[1:]:
        assert abs(l1 - l0) <= 1e-12 * abs(l0)
        assert np.abs(gf1 - gf0).max() <= 1e-9 * np.abs(gf0).max()
        assert np.abs(gq1 - gq0).max() <= 1e-9 * np.abs(gq0).max()


@gpu
def test_adjoint_field_and_weight_entries_vs_finite_differences():
    """Every field component and individual weights, central differences."""
    _require_gpu()
    p = SlabLaserProblem(_small_case())
    _, slab = p.nominal()
    f = _random_fields(p, seed=1)
    q = p.weights(slab).numpy()
    r = p.setup.region(f, q)
    loss, gf, gq = r.adjoint_energy(p.setup.nsteps, p.setup.every)
    r.close()

    def L(ff, qq):
        rr = p.setup.region(ff, qq)
        try:
            return rr.step(p.setup.nsteps)[-1].energy_e
        finally:
            rr.close()

    rng = np.random.default_rng(7)
    fscale = np.abs(f).max()
    gmax_f = np.abs(gf).max()
    checked = 0
    for c in range(6):
        # the two largest gradient entries of the component and one random interior entry
        flat = np.argsort(np.abs(gf[c]).ravel())[-2:]
        idx = [np.unravel_index(t, gf[c].shape) for t in flat]
        idx.append((rng.integers(2, 46), rng.integers(2, 26), rng.integers(2, 26)))
        for (i, j, k) in idx:
            h = H_REL * fscale
            fp = f.copy(); fp[c, i, j, k] += h
            fm = f.copy(); fm[c, i, j, k] -= h
            fd = (L(fp, q) - L(fm, q)) / (2 * h)
            assert _close(gf[c, i, j, k], fd, gmax_f), (c, i, j, k, gf[c, i, j, k], fd)
            checked += 1
    gmax_q = np.abs(gq).max()
    for s in list(np.argsort(np.abs(gq))[-3:]) + list(rng.integers(0, q.size, 3)):
        h = H_REL * abs(q[s]) if q[s] != 0 else H_REL * np.abs(q).max()
        qp_ = q.copy(); qp_[s] += h
        qm_ = q.copy(); qm_[s] -= h
        fd = (L(f, qp_) - L(f, qm_)) / (2 * h)
        assert _close(gq[s], fd, gmax_q), (s, gq[s], fd)
        checked += 1
    assert checked == 24


@gpu
def test_all_parameters_vs_finite_differences():
    """The 3 slab parameters and the 64 complex Gauss-Hermite coefficients
    (real and imaginary parts) through torch.autograd."""
    _require_gpu()
    p = SlabLaserProblem(_small_case())
    coef, slab = p.nominal()
    # a generic point: every mode present
    gen = torch.Generator().manual_seed(5)
    coef = coef + 0.25 * p.case.a0 * torch.complex(torch.randn(8, 8, generator=gen, dtype=torch.float64),
                                      torch.randn(8, 8, generator=gen, dtype=torch.float64))
    coef.requires_grad_(True)
    slab.requires_grad_(True)
    with torch.no_grad():
        r = p.setup.region(p.fields(coef).numpy(), p.weights(slab).numpy())
        r.step(p.setup.nsteps)
        assert r.count(0) == p.n_particles  # nothing erased: the loss is smooth here
        r.close()
    loss = p.loss(coef, slab)
    loss.backward()
    g_slab = slab.grad.numpy()
    g_coef = coef.grad.numpy()  # dL/dRe + i dL/dIm
    c0, s0 = coef.detach(), slab.detach()
    for t in range(3):
        h = H_REL * abs(s0[t].item())
        sp_, sm_ = s0.clone(), s0.clone()
        sp_[t] += h
        sm_[t] -= h
        fd = (p.loss_value(c0, sp_) - p.loss_value(c0, sm_)) / (2 * h)
        assert _close(g_slab[t], fd, np.abs(g_slab).max()), (t, g_slab[t], fd)
    gmax = np.abs(g_coef).max()
    h = H_REL * p.case.a0
    for m in range(8):
        for n in range(8):
            for part, unit in ((0, 1.0), (1, 1j)):
                cp_, cm_ = c0.clone(), c0.clone()
                cp_[m, n] += h * unit
                cm_[m, n] -= h * unit
                fd = (p.loss_value(cp_, s0) - p.loss_value(cm_, s0)) / (2 * h)
                ga = g_coef[m, n].real if part == 0 else g_coef[m, n].imag
                assert _close(ga, fd, gmax), (m, n, part, ga, fd)


@gpu
def test_mixed_forward_loss_close_to_fp64():
    _require_gpu()
    p = SlabLaserProblem(_small_case())
    coef, slab = p.nominal()
    l64 = p.loss_value(coef, slab, "fp64")
    l32 = p.loss_value(coef, slab, "mixed")
    assert abs(l32 - l64) <= 1e-4 * abs(l64)


@gpu
def test_mixed_adjoint_close_to_fp64_adjoint():
    """Mixed precision: the FP64 adjoint along the FP32 trajectory agrees
    with the FP64 adjoint to the trajectories' distance (here 1e-3 of each
    gradient's largest entry), for the fields, the weights and the 67
    parameters through the torch binding."""
    _require_gpu()
    p64 = SlabLaserProblem(_small_case())
    p32 = SlabLaserProblem(_small_case(), precision="mixed")
    _, slab = p64.nominal()
    f = _random_fields(p64)
    q = p64.weights(slab).numpy()
    out = {}
    for name, p in (("fp64", p64), ("mixed", p32)):
        r = p.setup.region(f, q)
        out[name] = r.adjoint_energy(p.setup.nsteps, p.setup.every)
        r.close()
    (l64, gf64, gq64), (l32, gf32, gq32) = out["fp64"], out["mixed"]
    assert abs(l32 - l64) <= 1e-4 * abs(l64)
    assert np.abs(gf32 - gf64).max() <= 1e-3 * np.abs(gf64).max()
    assert np.abs(gq32 - gq64).max() <= 1e-3 * np.abs(gq64).max()
    grads = {}
    for name, p in (("fp64", p64), ("mixed", p32)):
        coef, slab = p.nominal()
        coef.requires_grad_(True)
        slab.requires_grad_(True)
        p.loss(coef, slab).backward()
        grads[name] = (coef.grad.clone(), slab.grad.clone())
    for a, b in zip(grads["mixed"], grads["fp64"]):
        assert torch.abs(a - b).max() <= 1e-3 * torch.abs(b).max()


@gpu
def test_adjoint_rejects_unsupported_configurations():
    _require_gpu()
    from quill_b200.api import QPError, Region
    for kw in (dict(pusher="vay"), dict(solver="ndfx")):
        r = Region(20, 12, 12, 0.39, 0.39, 0.39, 0.19, **kw)
        r.set_fields(*np.zeros((6, 20, 12, 12)))
        r.init_boundaries()
        with pytest.raises(QPError):
            r.adjoint_energy(2, 1)
        r.close()
    r = Region(20, 12, 12, 0.39, 0.39, 0.39, 0.19)
    r.set_fields(*np.zeros((6, 20, 12, 12)))
    with pytest.raises(QPError):  # init_boundaries has not run
        r.adjoint_energy(2, 1)
    r.close()
