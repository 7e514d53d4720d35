"""Whose energy drift: the GPU step against the reference's own code on the
benchmark's throughput physics (configuration 5's plasma: 0.05 n_cr, 4
electrons per cell, 10 keV, dx = lambda/20, dt = dx/2, FDTD + Boris, a0 = 20
pulse) on a 32^3 box the reference steps 1000 times in seconds.

The closed balance is the total energy of the `energy` output (fields +
particles) plus the energy of the particles erased so far: on the reference
with catching on (update_energy_deleted, low-level.cpp:286-313), on the GPU
with qp_set_erased_tracking.  With the reference-order deposition the GPU
state is the reference's bit for bit, so the two balances agree to the
rounding of the diagnostic sums (1e-9 relative) at every checked step: the
residual drift of the balance is the scheme's own, not the GPU's.  The
default deposition (atomics) is reported beside them and held to 1e-2 of
the total: its state diverges from the reference's through the summation
order alone, so its balance follows the same scheme."""
import numpy as np
import pytest

from oracle import oracle as O
from quill_b200 import workloads as W
from tests.conftest import gpu_available

pytestmark = pytest.mark.gpu

FK = ("ex", "ey", "ez", "bx", "by", "bz")
STEPS = 1000
MARKS = (1, 100, 500, 1000)


@pytest.fixture(autouse=True)
def _need():
    if not gpu_available():
        pytest.skip("no CUDA device")
    if not O.available("ref", "parity"):
        pytest.skip("compiled reference (oracle/_ref) missing")


def _case():
    return W.scaled(W.config("cfg5_512_fdtd_boris"), 32, 32, 32, steps=STEPS)


def _ref_balance(case, fields, parts):
    reg = O.Region(case.nx, case.ny, case.nz, case.dx, case.dx, case.dx, case.dt, solver=0, pusher=1, kind="ref")
    reg.set_catching(True)
    try:
        reg.set_fields(*[fields[k] for k in FK])
        reg.init_boundaries()
        reg.add_particles(parts[0])
        out = {}
        for step in range(1, STEPS + 1):
            d = reg.step(1)[0]
            if step in MARKS:
                out[step] = float(d[6] + d[7] + d[8] + d[9] + reg.energy_deleted().sum())
        return out
    finally:
        reg.set_catching(False)


def _gpu_balance(case, fields, parts, ordered):
    from quill_b200.api import Region
    reg = Region(case.nx, case.ny, case.nz, case.dx, case.dx, case.dx, case.dt, species_cmr=(-1.0,),
                 solver="fdtd", pusher="boris")
    reg.set_fields(*[fields[k] for k in FK])
    reg.init_boundaries()
    reg.add_particles(0, parts[0])
    reg.set_erased_tracking(True)
    if ordered:
        reg.set_ordered_current(True)
    out, lost = {}, 0.0
    for step in range(1, STEPS + 1):
        d = reg.step(1)[0]
        lost += d.energy_erased
        if step in MARKS:
            out[step] = d.total_energy() + lost
    reg.close()
    return out


def test_closed_energy_balance_is_the_references():
    case = _case()
    fields, parts = W.build(case)
    ref = _ref_balance(case, fields, parts)
    ordered = _gpu_balance(case, fields, parts, True)
    atomic = _gpu_balance(case, fields, parts, False)
    w0 = ref[1]
    drift = {name: {s: (v[s] - w0) / w0 for s in MARKS} for name, v in
             (("reference", ref), ("gpu_reference_order", ordered), ("gpu_atomic", atomic))}
    print("closed-balance drift relative to step 1:", drift)
    for s in MARKS:
        assert abs(ordered[s] - ref[s]) <= 1e-9 * abs(ref[s]), (s, ordered[s], ref[s])
        assert abs(atomic[s] - ref[s]) <= 1e-2 * abs(ref[s]), (s, atomic[s], ref[s])
