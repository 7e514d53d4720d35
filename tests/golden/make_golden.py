"""Generate the golden vectors in this folder from the reference's own
sources (oracle/_ref, built by `make -C oracle ref`), parity build.

    python tests/golden/make_golden.py

Each case: a small grid with a laser-like field plus noise, electrons,
positrons, ions and photons (some loaded in the p_boundary layers), stepped
3 times; stores the inputs, the fields, particles (traversal order) and
diagnostics after every step.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from tests._cases import PUSHER_ID, SOLVER_ID, all_particles, small_case  # noqa: E402

CASES = [("fdtd", "boris", 0.5), ("ndfx", "vay", 0.5), ("five_point", "boris", 0.3)]
SPECIES = (-1.0, 1.0, 1 / 1836.15, 0.0)
STEPS = 3


def generate(solver, pusher, dtdx):
    case, fields, parts = small_case(solver, pusher, n=(12, 11, 10), ppc=1, dt_over_dx=dtdx, species=SPECIES,
                                     loaded_in_boundary=True, seed=11)
    reg = O.Region(case.nx, case.ny, case.nz, case.dx, case.dx, case.dx, case.dt, solver=SOLVER_ID[solver],
                   pusher=PUSHER_ID[pusher], icmr=(1 / 1836.15,), seed=7, kind="ref")
    fk = ("ex", "ey", "ez", "bx", "by", "bz")
    reg.set_fields(*[fields[k] for k in fk])
    reg.init_boundaries()
    ap = all_particles(parts)
    ap["chi"] = np.zeros(ap["x"].size)
    reg.add_particles(ap)
    out = {"grid": np.array([case.nx, case.ny, case.nz]), "dx": case.dx, "dt": case.dt,
           "solver": SOLVER_ID[solver], "pusher": PUSHER_ID[pusher], "external_bz": 0.3}
    for k in fk:
        out["in_" + k] = fields[k]
    for k in O.PARTICLE_KEYS:
        out["in_p_" + k] = ap[k]
    for s in range(STEPS):
        d = reg.step(1, external_bz=0.3)[0]
        f = reg.get_fields()
        p = reg.get_particles()
        out[f"s{s}_fields"] = f
        out[f"s{s}_diag"] = d
        for k in O.PARTICLE_KEYS:
            out[f"s{s}_p_{k}"] = p[k]
        out[f"s{s}_p_cell"] = p["cell"]
    return out


if __name__ == "__main__":
    if not O.available("ref", "parity"):
        raise SystemExit("build the reference first: make -C oracle ref")
    for solver, pusher, dtdx in CASES:
        out = generate(solver, pusher, dtdx)
        path = os.path.join(HERE, f"golden_{solver}_{pusher}.npz")
        np.savez_compressed(path, **out)
        print(path, os.path.getsize(path))
