"""Gradients of the final electron kinetic energy with respect to the initial
state, through the FP64 QED-off step (FDTD solver, Boris pusher).

`FinalElectronEnergy` is a torch.autograd.Function over the library's
hand-written discrete adjoint (`qp_adjoint_energy`): its forward runs the
region for `nsteps` steps and returns L = energy_e after the last step
(compute_energy's electron term, fout.cpp:87-138, normalised as
main.cpp:2326-2327); its backward returns the exact gradients of that
discrete computation with respect to the six loaded field planes and the
electrons' weights q.  The library saves the state every `every` steps and
re-runs each segment once for the backward sweep.

`SlabLaserProblem` is the differentiable workload around it (no reference
counterpart; the reference has no density profile of this form and no
adjoint):
  * plasma: a tanh slab n(x) = h/2 [tanh((x - c + w/2)/L) - tanh((x - c - w/2)/L)]
    (x in cells, height h in n_cr, centre c and width w in cells, fixed edge
    length L), carried by the weights q = -n(x)/ppc of electrons at fixed
    positions (the fill_cell_by_particles weight rule, init.cpp:402-414);
  * laser: an initial y-polarised pulse with a cos^2 envelope along x and a
    transverse envelope of N x N complex Gauss-Hermite coefficients c_mn,
    Ey = env(x) Re[sum_mn c_mn h_m(sqrt2 y/w) h_n(sqrt2 z/w) exp(-(y^2+z^2)/w^2)
    exp(i (x - x_c))], Bz likewise at the staggered Bz positions (h_m the
    normalised Hermite functions).
Its 3 + N^2 parameters are ordinary torch leaves; autograd chains the
adjoint's field and weight gradients through both maps.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np
import torch

from .api import Region

TWO_PI = 2.0 * math.pi


@dataclasses.dataclass
class SlabLaserCase:
    """Shapes of the adjoint workload.  The long axis is x, the laser's
    propagation axis, so that the slab centre (128 cells) lies inside."""
    nx: int = 256
    ny: int = 128
    nz: int = 128
    dx_lambda: float = 1 / 16
    dt_over_dx: float = 0.5
    nsteps: int = 400
    every: int = 32
    ppc: int = 4
    height: float = 0.5       # n / n_cr
    centre: float = 128.0     # cells
    width: float = 20.0       # cells
    edge: float = 2.0         # tanh edge length, cells (fixed)
    margin: float = 4.0       # particles fill [c - w/2 - margin*edge, c + w/2 + margin*edge)
    transverse_gap: int = 0   # cells kept free of particles inside each transverse boundary
    a0: float = 5.0
    fwhm_lambda: float = 2.0
    waist_lambda: float = 3.0
    n_modes: int = 8
    lambda_cm: float = 1e-4
    seed: int = 0

    @property
    def dx(self) -> float:
        return self.dx_lambda * TWO_PI

    @property
    def dt(self) -> float:
        return self.dt_over_dx * self.dx


class _Setup:
    """Non-differentiable part of a run: grid, particles' positions and
    momenta (traversal order), step count."""

    def __init__(self, shape, dx, dt, lambda_cm, particles: dict, nsteps: int, every: int,
                 external_bz: float = 0.0, device: int = 0, precision: str = "fp64"):
        self.shape = tuple(shape)
        self.dx, self.dt, self.lambda_cm = dx, dt, lambda_cm
        self.particles = particles
        self.nsteps, self.every = nsteps, every
        self.external_bz = external_bz
        self.device = device
        self.precision = precision

    def region(self, fields: np.ndarray, q: np.ndarray, precision=None) -> Region:
        precision = self.precision if precision is None else precision
        nx, ny, nz = self.shape
        r = Region(nx, ny, nz, self.dx, self.dx, self.dx, self.dt, species_cmr=(-1.0,), lambda_cm=self.lambda_cm,
                   solver="fdtd", pusher="boris", precision=precision, device=self.device)
        r.set_fields(*fields)
        r.init_boundaries()
        parts = dict(self.particles)
        parts["q"] = q
        r.add_particles(0, parts)
        return r


class FinalElectronEnergy(torch.autograd.Function):
    """L(fields, q) = energy_e after setup.nsteps steps.

    fields: float64 tensor (6, nx, ny, nz), Ex Ey Ez Bx By Bz as loaded;
    q: float64 tensor (n,), electron weights in traversal order (positions
    sorted by cell; the order inside a cell is kept).  With
    setup.precision == "mixed" the forward runs in mixed precision and the
    gradient is the FP64 adjoint along that trajectory."""

    @staticmethod
    def forward(ctx, fields: torch.Tensor, q: torch.Tensor, setup: _Setup):
        f_np = fields.detach().to("cpu", torch.float64).contiguous().numpy()
        q_np = q.detach().to("cpu", torch.float64).contiguous().numpy()
        need = ctx.needs_input_grad[0] or ctx.needs_input_grad[1]
        r = setup.region(f_np, q_np)
        try:
            if need:
                loss, gf, gq = r.adjoint_energy(setup.nsteps, setup.every, setup.external_bz)
            else:
                loss = r.step(setup.nsteps, setup.external_bz)[-1].energy_e
                gf = gq = None
        finally:
            r.close()
        if need:
            ctx.save_for_backward(torch.from_numpy(gf).to(fields.device), torch.from_numpy(gq).to(q.device))
        return fields.new_tensor(loss)

    @staticmethod
    def backward(ctx, grad_out):
        gf, gq = ctx.saved_tensors
        return grad_out * gf, grad_out * gq, None


def hermite_functions(u: torch.Tensor, n: int) -> torch.Tensor:
    """h_m(u) = H_m(u) / sqrt(2^m m!) for m < n (physicists' Hermite
    polynomials by the three-term recurrence), stacked along dim 0."""
    out = [torch.ones_like(u)]
    if n > 1:
        out.append(2.0 * u / math.sqrt(2.0))
    for m in range(1, n - 1):
        # H_{m+1} = 2u H_m - 2m H_{m-1}, rescaled to the normalised form
        out.append((2.0 * u * out[m] * math.sqrt(2.0 ** m * math.factorial(m))
                    - 2.0 * m * out[m - 1] * math.sqrt(2.0 ** (m - 1) * math.factorial(m - 1)))
                   / math.sqrt(2.0 ** (m + 1) * math.factorial(m + 1)))
    return torch.stack(out)


class SlabLaserProblem:
    """The tanh-slab / Gauss-Hermite-laser gradient problem on one GPU."""

    def __init__(self, case: SlabLaserCase, device: int = 0, precision: str = "fp64"):
        self.case = case
        c = case
        rng = np.random.default_rng(c.seed)
        x_lo = max(1, int(math.floor(c.centre - 0.5 * c.width - c.margin * c.edge)))
        x_hi = min(c.nx - 3, int(math.ceil(c.centre + 0.5 * c.width + c.margin * c.edge)))
        gap = c.transverse_gap
        ii, jj, kk = np.meshgrid(np.arange(x_lo, x_hi), np.arange(1 + gap, c.ny - 2 - gap),
                                 np.arange(1 + gap, c.nz - 2 - gap), indexing="ij")
        ci = np.repeat(ii.ravel(), c.ppc).astype(np.float64)
        cj = np.repeat(jj.ravel(), c.ppc).astype(np.float64)
        ck = np.repeat(kk.ravel(), c.ppc).astype(np.float64)
        m = ci.size
        zeros = np.zeros(m)
        self.particles = {"x": ci + rng.random(m), "y": cj + rng.random(m), "z": ck + rng.random(m),
                          "ux": zeros, "uy": zeros.copy(), "uz": zeros.copy(), "g": np.ones(m)}
        self.setup = _Setup((c.nx, c.ny, c.nz), c.dx, c.dt, c.lambda_cm, self.particles, c.nsteps, c.every,
                            device=device, precision=precision)
        self._x = torch.from_numpy(self.particles["x"])
        # laser geometry (cells): cos^2 half-length from the FWHM as the
        # reference's f_init_cos converts it (init.cpp:34-37)
        self.xs = 0.849 * c.fwhm_lambda * TWO_PI * 2 * math.sqrt(TWO_PI) / 3.0 / c.dx
        self.xc = self.xs + 2.0
        self.w = c.waist_lambda * TWO_PI / c.dx

    @property
    def n_particles(self) -> int:
        return self._x.numel()

    def nominal(self):
        """(coef, slab): the fundamental mode at a0 and the nominal slab."""
        c = self.case
        coef = torch.zeros(c.n_modes, c.n_modes, dtype=torch.complex128)
        coef[0, 0] = c.a0
        slab = torch.tensor([c.height, c.centre, c.width], dtype=torch.float64)
        return coef, slab

    def weights(self, slab: torch.Tensor) -> torch.Tensor:
        """q = -n(x)/ppc for the tanh slab (height, centre, width)."""
        h, cen, wid = slab[0], slab[1], slab[2]
        L = self.case.edge
        x = self._x.to(slab.device)
        n = 0.5 * h * (torch.tanh((x - cen + 0.5 * wid) / L) - torch.tanh((x - cen - 0.5 * wid) / L))
        return -n / self.case.ppc

    def fields(self, coef: torch.Tensor) -> torch.Tensor:
        """(6, nx, ny, nz) initial fields of the Gauss-Hermite pulse."""
        c = self.case
        dev = coef.device
        nmod = c.n_modes
        i = torch.arange(c.nx, dtype=torch.float64, device=dev)
        j = torch.arange(c.ny, dtype=torch.float64, device=dev)
        k = torch.arange(c.nz, dtype=torch.float64, device=dev)
        # Ey at (i, j+1/2, k), Bz at (i+1/2, j+1/2, k)
        yv = j + 0.5 - 0.5 * c.ny
        zv = k - 0.5 * c.nz
        hy = hermite_functions(math.sqrt(2.0) * yv / self.w, nmod)  # (M, ny)
        hz = hermite_functions(math.sqrt(2.0) * zv / self.w, nmod)  # (M, nz)
        gauss = torch.exp(-(yv[:, None] ** 2 + zv[None, :] ** 2) / (self.w * self.w))
        trans = torch.einsum("mn,mj,nk->jk", coef, hy.to(coef.dtype), hz.to(coef.dtype)) * gauss

        def wave(xp):
            a = (xp - self.xc) / self.xs
            env = torch.where(a.abs() < 1, torch.cos(0.5 * math.pi * a) ** 2, torch.zeros_like(a))
            ph = torch.polar(torch.ones_like(xp), (xp - self.xc) * c.dx)
            return env[:, None, None] * (ph[:, None, None] * trans[None]).real

        zero = torch.zeros(c.nx, c.ny, c.nz, dtype=torch.float64, device=dev)
        ey = wave(i)
        bz = wave(i + 0.5)
        return torch.stack([zero, ey, zero, zero, zero, bz])

    def loss(self, coef: torch.Tensor, slab: torch.Tensor) -> torch.Tensor:
        return FinalElectronEnergy.apply(self.fields(coef), self.weights(slab), self.setup)

    def loss_value(self, coef: torch.Tensor, slab: torch.Tensor, precision: str | None = None) -> float:
        """Forward only (FP64 or mixed precision; the problem's by default),
        no gradients."""
        with torch.no_grad():
            f = self.fields(coef).cpu().numpy()
            q = self.weights(slab).cpu().numpy()
        r = self.setup.region(f, q, precision=precision)
        try:
            return r.step(self.setup.nsteps, self.setup.external_bz)[-1].energy_e
        finally:
            r.close()


def _main(argv=None):
    """Time one loss + gradient evaluation of the adjoint workload and check
    selected parameters against central finite differences of the FP64
    forward (h = 1e-6 relative).  Prints one JSON line."""
    import argparse
    import json
    import time

    ap = argparse.ArgumentParser(description=_main.__doc__)
    ap.add_argument("--grid", type=int, nargs=3, default=None, help="nx ny nz (default 256 128 128)")
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--every", type=int, default=None)
    ap.add_argument("--transverse-gap", type=int, default=0)
    ap.add_argument("--check", type=int, default=4, help="Gauss-Hermite coefficients checked (plus the 3 slab parameters)")
    ap.add_argument("--a0", type=float, default=None)
    a = ap.parse_args(argv)
    case = SlabLaserCase(transverse_gap=a.transverse_gap)
    if a.grid:
        case.nx, case.ny, case.nz = a.grid
        case.centre = 0.5 * case.nx
    if a.steps:
        case.nsteps = a.steps
    if a.every:
        case.every = a.every
    if a.a0:
        case.a0 = a.a0
    p = SlabLaserProblem(case)
    coef, slab = p.nominal()
    coef.requires_grad_(True)
    slab.requires_grad_(True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    loss = p.loss(coef, slab)
    loss.backward()
    t_grad = time.perf_counter() - t0
    t0 = time.perf_counter()
    l_fwd = p.loss_value(coef.detach(), slab.detach())
    t_fwd = time.perf_counter() - t0
    # particles erased during the run make the loss jump: the difference
    # quotients are only meaningful when this is 0
    with torch.no_grad():
        r = p.setup.region(p.fields(coef).numpy(), p.weights(slab).numpy())
        r.step(case.nsteps)
        erased = p.n_particles - r.count(0)
        r.close()
    c0, s0 = coef.detach(), slab.detach()
    errs = {}
    for t, name in enumerate(("height", "centre", "width")):
        h = 1e-6 * abs(s0[t].item())
        sp_, sm_ = s0.clone(), s0.clone()
        sp_[t] += h
        sm_[t] -= h
        fd = (p.loss_value(c0, sp_) - p.loss_value(c0, sm_)) / (2 * h)
        errs[name] = {"adjoint": slab.grad[t].item(), "fd": fd}
    h = 1e-6 * case.a0
    for m in range(min(a.check, case.n_modes * case.n_modes)):
        mm, nn = divmod(m, case.n_modes)
        cp_, cm_ = c0.clone(), c0.clone()
        cp_[mm, nn] += h
        cm_[mm, nn] -= h
        fd = (p.loss_value(cp_, s0) - p.loss_value(cm_, s0)) / (2 * h)
        errs[f"Re c{mm}{nn}"] = {"adjoint": coef.grad[mm, nn].real.item(), "fd": fd}
    gmax = max(abs(v["adjoint"]) for v in errs.values())
    for v in errs.values():
        v["rel_err"] = abs(v["adjoint"] - v["fd"]) / max(abs(v["fd"]), 1e-300)
    print(json.dumps({"workload": f"slab + Gauss-Hermite laser, {case.nx}x{case.ny}x{case.nz} cells, "
                                  f"{p.n_particles} electrons, {case.nsteps} steps, checkpoint every {case.every}",
                      "loss": loss.item(), "loss_forward_only": l_fwd, "seconds_loss_and_gradient": t_grad,
                      "seconds_forward": t_fwd, "particles_erased": erased, "max_abs_gradient": gmax,
                      "checks": errs}))


if __name__ == "__main__":
    _main()
