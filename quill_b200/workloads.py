"""Synthetic initial states in the shapes of the benchmark configurations.

All quantities are in the reference's normalised units (lengths c/omega,
time 1/omega, fields m c omega / e, positions in cell units).  With the
wavelength lambda = 1 um, one wavelength is 2*pi in length units.

Plasma macro-particle weight follows fill_cell_by_particles
(init.cpp:402-414): q = +-n / ppc with n in units of the critical density.
The laser is an initial field (the reference has no injector, init.cpp:6-385):
a pulse with a cos^2 longitudinal envelope and a Gaussian transverse profile,
placed just inside x = 0 and moving towards +x.  Its widths use the
conversion of the reference's f_init_cos inputs: xsigma = 0.849 * FWHM
(intensity), ysigma = zsigma = waist.

These states are synthetic stand-ins for the configurations; no data set is
involved.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

TWO_PI = 2.0 * math.pi
PROTON_CMR = 1.0 / 1836.15
KEV_THETA = 1.957e-3  # T = 1 keV in units of m c^2


@dataclasses.dataclass
class SpeciesSpec:
    cmr: float
    ppc: int
    density: str = "uniform"          # uniform | slab | ramp | sphere
    n0: float = 0.1                   # n / n_cr
    x_range: tuple = (0.0, 1.0)       # fraction of nx (slab)
    ramp_cells: int = 40
    theta: float = 0.0                # temperature in m c^2 (0 = cold)
    radius_lambda: float = 2.0


@dataclasses.dataclass
class LaserSpec:
    a0: float
    fwhm_lambda: float
    waist_lambda: float
    polarization: str = "linear"      # linear | circular
    counter: bool = False             # add a mirror pulse travelling towards -x


@dataclasses.dataclass
class Case:
    name: str
    nx: int
    ny: int
    nz: int
    dx_lambda: float
    dt_over_dx: float
    solver: str
    pusher: str
    steps: int
    species: list
    laser: LaserSpec | None
    qed: bool = False
    seed: int = 0

    @property
    def dx(self) -> float:
        return self.dx_lambda * TWO_PI

    @property
    def dt(self) -> float:
        return self.dt_over_dx * self.dx


def config(name: str) -> Case:
    """Benchmark configurations (BASELINE shapes)."""
    if name == "cfg1_64_fdtd_boris":
        return Case(name, 64, 64, 64, 1 / 16, 0.5, "fdtd", "boris", 200,
                    [SpeciesSpec(-1.0, 2, "slab", 0.1, (16 / 64, 48 / 64), theta=KEV_THETA)],
                    LaserSpec(10.0, 5.0, 3.0, "linear"))
    if name == "cfg2_256_ndfx_vay":
        return Case(name, 256, 256, 256, 1 / 20, 0.5, "ndfx", "vay", 500,
                    [SpeciesSpec(-1.0, 8, "ramp", 1.0, ramp_cells=40),
                     SpeciesSpec(PROTON_CMR, 8, "ramp", 1.0, ramp_cells=40)],
                    LaserSpec(50.0, 8.0, 4.0, "circular"))
    if name == "cfg3_256_fivepoint_vay_qed":
        return Case(name, 256, 256, 256, 1 / 32, 0.3, "five_point", "vay", 600,
                    [SpeciesSpec(-1.0, 4, "sphere", 1e-2, radius_lambda=2.0),
                     SpeciesSpec(PROTON_CMR, 4, "sphere", 1e-2, radius_lambda=2.0)],
                    LaserSpec(1500.0, 10.0, 3.0, "circular", counter=True), qed=True)
    if name == "cfg4_128x128x256_fdtd_boris":
        return Case(name, 128, 128, 256, 1 / 16, 0.5, "fdtd", "boris", 400,
                    [SpeciesSpec(-1.0, 4, "uniform", 0.5)], LaserSpec(5.0, 5.0, 3.0, "linear"))
    if name == "cfg5_512_fdtd_boris":
        return Case(name, 512, 512, 512, 1 / 20, 0.5, "fdtd", "boris", 1000,
                    [SpeciesSpec(-1.0, 4, "uniform", 0.05, theta=10 * KEV_THETA)],
                    LaserSpec(20.0, 6.0, 8.0, "linear"))
    raise KeyError(name)


def scaled(case: Case, nx: int, ny: int, nz: int, steps: int | None = None) -> Case:
    """The same physics on a smaller grid (same dx, dt, densities, ppc)."""
    c = dataclasses.replace(case, nx=nx, ny=ny, nz=nz)
    if steps is not None:
        c.steps = steps
    return c


def _profile(sp: SpeciesSpec, case: Case, ci: np.ndarray, cj: np.ndarray, ck: np.ndarray) -> np.ndarray:
    nx, ny, nz = case.nx, case.ny, case.nz
    if sp.density == "uniform":
        return np.full(ci.shape, sp.n0)
    if sp.density == "slab":
        lo, hi = sp.x_range
        return np.where((ci >= lo * nx) & (ci < hi * nx), sp.n0, 0.0)
    if sp.density == "ramp":
        # linear ramp from 0 to n0 over ramp_cells starting a quarter into x
        x0 = nx // 4
        return np.clip((ci - x0 + 0.5) / sp.ramp_cells, 0.0, 1.0) * sp.n0 * (ci >= x0)
    if sp.density == "sphere":
        r = sp.radius_lambda / case.dx_lambda
        d2 = (ci + 0.5 - nx / 2) ** 2 + (cj + 0.5 - ny / 2) ** 2 + (ck + 0.5 - nz / 2) ** 2
        return np.where(d2 <= r * r, sp.n0, 0.0)
    raise KeyError(sp.density)


def make_particles(case: Case, sp: SpeciesSpec, rng: np.random.Generator, i_range=None) -> dict:
    """Particles in traversal order (cells lexicographic), ppc per occupied
    cell, uniform-random positions inside the cell, Maxwellian or cold
    momenta.  Only cells the reference keeps (is_inside: 1..n-3 per axis,
    plist.cpp:42-48) are filled; i_range = (a, b) limits them to the
    x-layers [a, b)."""
    nx, ny, nz = case.nx, case.ny, case.nz
    ia, ib = (1, nx - 2) if i_range is None else i_range
    ii, jj, kk = np.meshgrid(np.arange(ia, ib), np.arange(1, ny - 2), np.arange(1, nz - 2), indexing="ij")
    ii, jj, kk = ii.ravel(), jj.ravel(), kk.ravel()
    n = _profile(sp, case, ii, jj, kk)
    occ = n > 0
    ii, jj, kk, n = ii[occ], jj[occ], kk[occ], n[occ]
    ppc = sp.ppc
    ci = np.repeat(ii, ppc).astype(np.float64)
    cj = np.repeat(jj, ppc).astype(np.float64)
    ck = np.repeat(kk, ppc).astype(np.float64)
    nn = np.repeat(n, ppc)
    m = ci.size
    x = ci + rng.random(m)
    y = cj + rng.random(m)
    z = ck + rng.random(m)
    if sp.theta > 0:
        s = math.sqrt(sp.theta)
        ux, uy, uz = (rng.standard_normal(m) * s for _ in range(3))
    else:
        ux = np.zeros(m); uy = np.zeros(m); uz = np.zeros(m)
    if sp.cmr == 0:
        g = np.sqrt(ux * ux + uy * uy + uz * uz)
    else:
        g = np.sqrt(1 + ux * ux + uy * uy + uz * uz)
    q = nn / ppc
    if sp.cmr < 0:
        q = -q
    return {"x": x, "y": y, "z": z, "ux": ux, "uy": uy, "uz": uz, "g": g, "q": q,
            "cmr": np.full(m, sp.cmr)}


def make_fields(case: Case, i0: int = 0, nxr: int | None = None) -> dict:
    """Initial E and B: the laser pulse (zero elsewhere).  With i0 / nxr,
    only the x-layers [i0, i0 + nxr) of the box (an x-slab region)."""
    nx, ny, nz = case.nx, case.ny, case.nz
    if nxr is None:
        nxr = nx
    shape = (nxr, ny, nz)
    f = {k: np.zeros(shape) for k in ("ex", "ey", "ez", "bx", "by", "bz")}
    L = case.laser
    if L is None:
        return f
    dx = case.dx
    k0 = 1.0  # wave number of the laser in omega/c units
    xs = 0.849 * L.fwhm_lambda * TWO_PI * 2 * math.sqrt(TWO_PI) / 3.0  # f_init_cos half-length (init.cpp:34-37)
    xs = min(xs, 0.45 * nx * dx)
    w = L.waist_lambda * TWO_PI
    xc = xs  # pulse centre one half-length inside x = 0

    def env(xpos):
        a = (xpos - xc) / xs
        return np.where(np.abs(a) < 1, np.cos(0.5 * math.pi * a) ** 2, 0.0)

    # staggered positions (cell units): Ey at (i, j+1/2, k), Ez at (i, j, k+1/2),
    # Bz at (i+1/2, j+1/2, k), By at (i+1/2, j, k+1/2)
    i = np.arange(i0, i0 + nxr)[:, None, None].astype(np.float64)
    j = np.arange(ny)[None, :, None].astype(np.float64)
    k = np.arange(nz)[None, None, :].astype(np.float64)

    def trans(jp, kp):
        r2 = ((jp - ny / 2) * dx) ** 2 + ((kp - nz / 2) * dx) ** 2
        return np.exp(-r2 / (w * w))

    def wave(xp, phase):
        xpos = xp * dx
        return L.a0 * env(xpos) * np.cos(k0 * (xpos - xc) + phase)

    pol = [1.0, 0.0] if L.polarization == "linear" else [1.0 / math.sqrt(2), 1.0 / math.sqrt(2)]
    f["ey"] = pol[0] * wave(i, 0.0) * trans(j + 0.5, k)
    f["bz"] = pol[0] * wave(i + 0.5, 0.0) * trans(j + 0.5, k)
    if pol[1]:
        f["ez"] = pol[1] * wave(i, -0.5 * math.pi) * trans(j, k + 0.5)
        f["by"] = -pol[1] * wave(i + 0.5, -0.5 * math.pi) * trans(j, k + 0.5)
    if L.counter:
        if nxr != nx:
            raise ValueError("counter-propagating pulse: whole box only")
        # mirror pulse: x -> nx-1-x, travelling towards -x (B changes sign)
        for key, sgn in (("ey", 1), ("ez", 1), ("by", -1), ("bz", -1)):
            f[key] = f[key] + sgn * f[key][::-1, :, :]
    return {kk_: np.ascontiguousarray(v) for kk_, v in f.items()}


def particle_layers(case: Case, sp: SpeciesSpec, rng: np.random.Generator, i0: int, nxr: int,
                    layers_per_chunk: int = 4):
    """Particles of the x-layers [i0, i0 + nxr) of the box (an x-slab region,
    positions in its frame: x - i0), in groups of layers, each in traversal
    order; the same plasma as make_particles (cells the reference keeps,
    ppc per occupied cell, uniform-random positions, Maxwellian or cold
    momenta)."""
    lo, hi = max(i0, 1), min(i0 + nxr, case.nx - 2)
    for a in range(lo, hi, layers_per_chunk):
        b = min(a + layers_per_chunk, hi)
        part = make_particles(case, sp, rng, i_range=(a, b))
        if part["x"].size:
            part["x"] = part["x"] - i0
            yield part


def build(case: Case):
    """(fields dict, list of particle dicts) for a case, seeded."""
    rng = np.random.default_rng(case.seed)
    fields = make_fields(case)
    parts = [make_particles(case, sp, rng) for sp in case.species]
    return fields, parts


# ---------------------------------------------------------------------------
# Device-side generation (torch on the GPU) of the same states, for sizes
# where host generation would dominate (the 512^3 configuration holds 5.4e8
# particles).  Same formulas as make_fields / make_particles; the random
# streams differ from numpy's.
# ---------------------------------------------------------------------------

def make_fields_torch(case: Case, device="cuda", i0: int = 0, nxr: int | None = None):
    """make_fields on the device; with i0 / nxr only the x-layers
    [i0, i0 + nxr) of the box (an x-slab region)."""
    import torch
    nx, ny, nz = case.nx, case.ny, case.nz
    if nxr is None:
        nxr = nx
    z0 = lambda: torch.zeros((nxr, ny, nz), dtype=torch.float64, device=device)
    f = {k: z0() for k in ("ex", "ey", "ez", "bx", "by", "bz")}
    L = case.laser
    if L is None:
        return f
    dx = case.dx
    xs = 0.849 * L.fwhm_lambda * TWO_PI * 2 * math.sqrt(TWO_PI) / 3.0
    xs = min(xs, 0.45 * nx * dx)
    w = L.waist_lambda * TWO_PI
    xc = xs
    i = torch.arange(i0, i0 + nxr, dtype=torch.float64, device=device)
    j = torch.arange(ny, dtype=torch.float64, device=device)
    k = torch.arange(nz, dtype=torch.float64, device=device)

    def wave(xp, phase):
        xpos = xp * dx
        a = (xpos - xc) / xs
        env = torch.where(a.abs() < 1, torch.cos(0.5 * math.pi * a) ** 2, torch.zeros_like(a))
        return L.a0 * env * torch.cos(xpos - xc + phase)

    def trans(jp, kp):
        ry = ((jp - ny / 2) * dx) ** 2
        rz = ((kp - nz / 2) * dx) ** 2
        return torch.exp(-(ry[:, None] + rz[None, :]) / (w * w))

    pol = [1.0, 0.0] if L.polarization == "linear" else [1.0 / math.sqrt(2), 1.0 / math.sqrt(2)]
    t_ey = trans(j + 0.5, k)
    f["ey"] = pol[0] * wave(i, 0.0)[:, None, None] * t_ey[None]
    f["bz"] = pol[0] * wave(i + 0.5, 0.0)[:, None, None] * t_ey[None]
    if pol[1]:
        t_ez = trans(j, k + 0.5)
        f["ez"] = pol[1] * wave(i, -0.5 * math.pi)[:, None, None] * t_ez[None]
        f["by"] = -pol[1] * wave(i + 0.5, -0.5 * math.pi)[:, None, None] * t_ez[None]
    if L.counter:
        if nxr != nx:
            raise ValueError("counter-propagating pulse: whole box only")
        for key, sgn in (("ey", 1), ("ez", 1), ("by", -1), ("bz", -1)):
            f[key] = f[key] + sgn * torch.flip(f[key], dims=(0,))
    return {kk: v.contiguous() for kk, v in f.items()}


def particle_chunks_torch(case: Case, sp: SpeciesSpec, planes_per_chunk=32, device="cuda", seed=0, i_range=None):
    """Yield particle dicts (torch float64 tensors on the device) for groups
    of x-planes, in traversal order, ppc per occupied cell; with i_range =
    (a, b) only the x-layers [a, b), positions in the frame of layer a (an
    x-slab region starting there)."""
    import torch
    nx, ny, nz = case.nx, case.ny, case.nz
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    jj, kk = torch.meshgrid(torch.arange(1, ny - 2, device=device), torch.arange(1, nz - 2, device=device),
                            indexing="ij")
    jj, kk = jj.reshape(-1), kk.reshape(-1)
    lo, hi = (1, nx - 2) if i_range is None else (max(1, i_range[0]), min(nx - 2, i_range[1]))
    shift = 0 if i_range is None else i_range[0]
    for i0 in range(lo, hi, planes_per_chunk):
        i1 = min(i0 + planes_per_chunk, hi)
        ii = torch.arange(i0, i1, device=device).repeat_interleave(jj.numel())
        cj = jj.repeat(i1 - i0)
        ck = kk.repeat(i1 - i0)
        n = torch.as_tensor(_profile(sp, case, ii.cpu().numpy(), cj.cpu().numpy(), ck.cpu().numpy()),
                            device=device) if sp.density != "uniform" else None
        if n is not None:
            occ = n > 0
            ii, cj, ck, n = ii[occ], cj[occ], ck[occ], n[occ]
        m = ii.numel() * sp.ppc
        if m == 0:
            continue
        rep = lambda t: t.repeat_interleave(sp.ppc).to(torch.float64)
        x = rep(ii) - shift + torch.rand(m, generator=gen, device=device, dtype=torch.float64)
        y = rep(cj) + torch.rand(m, generator=gen, device=device, dtype=torch.float64)
        z = rep(ck) + torch.rand(m, generator=gen, device=device, dtype=torch.float64)
        if sp.theta > 0:
            s = math.sqrt(sp.theta)
            ux, uy, uz = (torch.randn(m, generator=gen, device=device, dtype=torch.float64) * s for _ in range(3))
        else:
            ux = torch.zeros(m, device=device, dtype=torch.float64)
            uy = torch.zeros_like(ux)
            uz = torch.zeros_like(ux)
        g = torch.sqrt(1 + ux * ux + uy * uy + uz * uz) if sp.cmr != 0 else torch.sqrt(ux * ux + uy * uy + uz * uz)
        qv = (rep(n) if n is not None else torch.full((m,), sp.n0, device=device, dtype=torch.float64)) / sp.ppc
        if sp.cmr < 0:
            qv = -qv
        yield {"x": x, "y": y, "z": z, "ux": ux, "uy": uy, "uz": uz, "g": g, "q": qv}
