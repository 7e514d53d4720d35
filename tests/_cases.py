"""Small seeded cases shared by the parity tests (the configurations' physics
on grids the CPU checkers finish in seconds)."""
import numpy as np

from quill_b200 import workloads as W

SOLVER_ID = {"fdtd": 0, "ndfx": 1, "five_point": 2}
PUSHER_ID = {"vay": 0, "boris": 1}


def small_case(solver="fdtd", pusher="boris", n=(20, 18, 16), ppc=2, theta=0.02, a0=10.0, seed=1,
               species=(-1.0,), dx_lambda=1 / 16, dt_over_dx=0.5, density="uniform", n0=0.2,
               loaded_in_boundary=False):
    sp = [W.SpeciesSpec(c, ppc, density, n0, theta=theta if c != 0 else 0.0) for c in species]
    case = W.Case("small", n[0], n[1], n[2], dx_lambda, dt_over_dx, solver, pusher, 10, sp,
                  W.LaserSpec(a0, 1.0, 0.6, "linear"), seed=seed)
    fields, parts = W.build(case)
    rng = np.random.default_rng(seed + 100)
    # add a little noise so every stencil term is exercised
    for k in fields:
        fields[k] = fields[k] + 0.05 * a0 * rng.standard_normal(fields[k].shape)
    for sp_, p in zip(case.species, parts):
        if sp_.cmr == 0:
            # photons: random directions with gamma = |u|
            m = p["x"].size
            u = rng.standard_normal((3, m)) * 3.0
            p["ux"], p["uy"], p["uz"] = u
            p["g"] = np.sqrt((u * u).sum(0))
        else:
            # relativistic tail so that particles cross cells every step
            m = p["x"].size
            u = rng.standard_normal((3, m)) * 1.5
            p["ux"], p["uy"], p["uz"] = u
            p["g"] = np.sqrt(1 + (u * u).sum(0))
    if loaded_in_boundary:
        # a few particles in the p_boundary layers (erased on the first step)
        p = parts[0]
        extra = {k: v[:6].copy() for k, v in p.items()}
        extra["x"] = np.array([0.5, case.nx - 1.5, case.nx - 0.5, 3.5, 3.5, 3.5])
        extra["y"][3] = 0.25
        extra["z"][4] = case.nz - 1.75
        extra["y"][5] = case.ny - 2.5
        idx = np.argsort(((extra["x"].astype(int) * case.ny + extra["y"].astype(int)) * case.nz
                          + extra["z"].astype(int)), kind="stable")
        merged = {k: np.concatenate([p[k], extra[k][idx]]) for k in p}
        cells = ((merged["x"].astype(int) * case.ny + merged["y"].astype(int)) * case.nz + merged["z"].astype(int))
        o = np.argsort(cells, kind="stable")
        parts[0] = {k: v[o] for k, v in merged.items()}
    return case, fields, parts


def all_particles(parts):
    keys = parts[0].keys()
    cat = {k: np.concatenate([p[k] for p in parts]) for k in keys}
    return cat
