"""Pin the C restatement (oracle/qp_oracle.c) against the reference's own
sources compiled by `make -C oracle ref` (oracle/_ref): bit-for-bit equal
fields, particles (order included) and diagnostics, with the parity builds
of both (no fused multiply-add)."""
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle as O
from tests._cases import PUSHER_ID, SOLVER_ID, all_particles, small_case

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _ensure_port():
    if not O.available("port", "parity"):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True, capture_output=True)


needs_ref = pytest.mark.skipif(not O.available("ref", "parity"),
                               reason="reference not compiled here (make -C oracle ref)")


def _region(kind, case, icmr=()):
    return O.Region(case.nx, case.ny, case.nz, case.dx, case.dx, case.dx, case.dt,
                    solver=SOLVER_ID[case.solver], pusher=PUSHER_ID[case.pusher], icmr=icmr,
                    seed=7, kind=kind)


def _load(reg, fields, parts):
    reg.set_fields(fields["ex"], fields["ey"], fields["ez"], fields["bx"], fields["by"], fields["bz"])
    reg.init_boundaries()
    reg.add_particles(all_particles(parts))


@needs_ref
@pytest.mark.parametrize("solver", ["fdtd", "ndfx", "five_point"])
@pytest.mark.parametrize("pusher", ["boris", "vay"])
def test_port_equals_reference_steps(solver, pusher):
    _ensure_port()
    dtdx = 0.3 if solver == "five_point" else 0.5
    case, fields, parts = small_case(solver, pusher, dt_over_dx=dtdx, species=(-1.0, 1.0, 1 / 1836.15, 0.0),
                                     loaded_in_boundary=True)
    icmr = (1 / 1836.15,)
    ref = _region("ref", case, icmr)
    port = _region("port", case, icmr)
    _load(ref, fields, parts)
    _load(port, fields, parts)
    np.testing.assert_array_equal(ref.get_fields(), port.get_fields())
    for step in range(6):
        dr = ref.step(1, external_bz=0.3)
        dp = port.step(1, external_bz=0.3)
        pr, pp = ref.get_particles(), port.get_particles()
        assert pr["x"].size == pp["x"].size
        for k in O.PARTICLE_KEYS:
            np.testing.assert_array_equal(pr[k], pp[k], err_msg=f"step {step} {k}")
        np.testing.assert_array_equal(pr["cell"], pp["cell"])
        np.testing.assert_array_equal(ref.get_fields(), port.get_fields(), err_msg=f"step {step}")
        np.testing.assert_array_equal(dr, dp)


@needs_ref
def test_unit_functions_equal_reference():
    _ensure_port()
    rng = np.random.default_rng(3)
    for _ in range(200):
        st = np.r_[rng.standard_normal(3) * 5, 0.0]
        st[3] = np.sqrt(1 + (st[:3] ** 2).sum())
        e, b = rng.standard_normal(3) * 30, rng.standard_normal(3) * 30
        for pusher in (0, 1):
            a = O.push(pusher, -1.0, st, e, b, 0.2, kind="ref")
            c = O.push(pusher, -1.0, st, e, b, 0.2, kind="port")
            np.testing.assert_array_equal(a, c)
    case, fields, parts = small_case()
    ref, port = _region("ref", case), _region("port", case)
    _load(ref, fields, parts)
    _load(port, fields, parts)
    for _ in range(300):
        pos = rng.uniform(2, 12, 3)
        d = rng.uniform(-0.9, 0.9, 3)
        for r in (ref, port):
            r.zero_j()
        a = ref.jdeposition(pos, d, 0.37)
        c = port.jdeposition(pos, d, 0.37)
        np.testing.assert_array_equal(a, c)
        np.testing.assert_array_equal(ref.get_fields()[6:9], port.get_fields()[6:9])
        ea, ba = ref.gather(*pos)
        ec, bc = port.gather(*pos)
        np.testing.assert_array_equal(ea, ec)
        np.testing.assert_array_equal(ba, bc)
    # QED rates and the random stream
    for _ in range(300):
        e, b, u = rng.standard_normal(3) * 1e3, rng.standard_normal(3) * 1e3, rng.standard_normal(3) * 1e3
        g = float(np.sqrt(1 + (u * u).sum()))
        assert ref.chi(e, b, u, g) == port.chi(e, b, u, g)
        chi = float(rng.uniform(0.01, 3))
        r = float(rng.uniform(0, 1))
        assert ref.w(g, r, chi) == port.w(g, r, chi)
        assert ref.tilde_w(g, r, chi) == port.tilde_w(g, r, chi)
        e2 = rng.standard_normal(3) * 1e5
        assert ref.mathcal_W(e2, b) == port.mathcal_W(e2, b)
    for _ in range(500):
        assert ref.get_rand() == port.get_rand()


@needs_ref
@pytest.mark.parametrize("mode,ppd", [("ti", [0.3]), ("nl", [0.6, 0.4, 0.8, 0.5])])
def test_merging_equals_reference(mode, ppd):
    """spatial_region::pmerging (mc.cpp:202-462): the same particles deleted
    (one draw of the lagged-Fibonacci stream per particle, traversal order),
    the same rescaled weights, then the same steps."""
    _ensure_port()
    species = (-1.0, 1.0, 0.0, 1 / 1836.15)
    case, fields, parts = small_case(species=species, ppc=3)
    # weights spread over a decade so that "nl" prefers the light ones
    rng = np.random.default_rng(11)
    for p in parts:
        p["q"] = p["q"] * rng.uniform(0.3, 3.0, p["q"].size)
    ref, port = _region("ref", case, icmr=(1 / 1836.15,)), _region("port", case, icmr=(1 / 1836.15,))
    for r in (ref, port):
        _load(r, fields, parts)
        r.step(1)
    n0 = ref.count()
    for r in (ref, port):
        r.pmerging(mode, ppd)
    a, b = ref.get_particles(), port.get_particles()
    assert 0 < ref.count() < n0
    for k in a:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    dr, dp = ref.step(2), port.step(2)
    np.testing.assert_array_equal(dr, dp)
    np.testing.assert_array_equal(ref.get_fields(), port.get_fields())


@needs_ref
def test_moving_window_equals_reference():
    """spatial_region::moving_window (advance.cpp:389-454) between steps."""
    _ensure_port()
    species = (-1.0, 1 / 1836.15)
    case, fields, parts = small_case(species=species, ppc=2)
    ref, port = _region("ref", case, icmr=(1 / 1836.15,)), _region("port", case, icmr=(1 / 1836.15,))
    for r in (ref, port):
        _load(r, fields, parts)
    for _ in range(3):
        dr, dp = ref.step(1), port.step(1)
        np.testing.assert_array_equal(dr, dp)
        before = ref.get_particles()
        ynz = case.ny * case.nz
        ref.moving_window()
        port.moving_window()
        assert ref.count() == int(np.sum(before["cell"] >= ynz))
        np.testing.assert_array_equal(ref.get_particles()["x"], before["x"][before["cell"] >= ynz] - 1)
        a, b = ref.get_particles(), port.get_particles()
        for k in a:
            np.testing.assert_array_equal(a[k], b[k], err_msg=k)
        np.testing.assert_array_equal(ref.get_fields(), port.get_fields())
