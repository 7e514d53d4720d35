"""Particle tracks (start_tracking, main.cpp:1516-1612): a track number per
particle, carried through the pushes, the rebin's reordering, merging and
the moving window; particles that join later are untracked.

Photons move ballistically (no fields act on them), so a tracked photon's
position after n steps is its start plus n displacements computed with the
push's own operations, which identifies it exactly."""
import math

import numpy as np
import pytest

from tests.conftest import gpu_available

pytestmark = pytest.mark.gpu

N = (24, 20, 18)
DX = 2 * math.pi / 16
DT = 0.5 * DX


def _photons(m=6000, seed=2):
    rng = np.random.default_rng(seed)
    u = rng.standard_normal((3, m)) * 3.0
    p = {"x": rng.uniform(3, N[0] - 5, m), "y": rng.uniform(3, N[1] - 5, m), "z": rng.uniform(3, N[2] - 5, m),
         "ux": u[0], "uy": u[1], "uz": u[2], "g": np.sqrt((u * u).sum(0)), "q": rng.uniform(0.01, 0.1, m)}
    cells = (p["x"].astype(int) * N[1] + p["y"].astype(int)) * N[2] + p["z"].astype(int)
    o = np.argsort(cells, kind="stable")
    return {k: v[o] for k, v in p.items()}


def _region(precision="fp64"):
    from quill_b200.api import Region
    r = Region(*N, DX, DX, DX, DT, species_cmr=(0.0,), precision=precision)
    r.set_fields(*np.zeros((6,) + N))
    r.init_boundaries()
    return r


def _mark(r, cells):
    first = r.first_in_cells(0, cells)
    pos = first[first >= 0]
    r.set_track_numbers(0, pos, np.arange(1, pos.size + 1))
    return pos


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_tracks_follow_their_particles(precision):
    if not gpu_available():
        pytest.skip("needs a CUDA device")
    p = _photons()
    r = _region(precision)
    r.add_particles(0, p)
    r.set_tracking(True)
    before = r.get_particles(0)
    rng = np.random.default_rng(9)
    cells = np.unique(rng.choice(before["cell"], 40, replace=False))
    pos = _mark(r, cells)
    assert pos.size == cells.size
    nsteps = 6
    r.step(nsteps)
    t = r.get_tracked(0)
    r.close()
    assert t["trn"].size > pos.size // 2
    for k, trn in enumerate(t["trn"]):
        s = pos[trn - 1]
        x = np.array([before["x"][s], before["y"][s], before["z"][s]])
        u = np.array([before["ux"][s], before["uy"][s], before["uz"][s]])
        g = before["g"][s]
        for _ in range(nsteps):  # the push's operations (containers.cpp:58-67, advance.cpp:281-284)
            tt = DT / g
            x = x + (u * tt) / DX
        got = np.array([t["x"][k], t["y"][k], t["z"][k]])
        if precision == "fp64":
            assert np.array_equal(got, x), (trn, got, x)
        else:
            assert np.abs(got - x).max() < 1e-4
        assert t["q"][k] == before["q"][s] if precision == "fp64" else abs(t["q"][k] - before["q"][s]) < 1e-7


def test_tracks_survive_merging_and_the_moving_window():
    if not gpu_available():
        pytest.skip("needs a CUDA device")
    p = _photons(seed=3)
    r = _region()
    r.add_particles(0, p)
    r.set_tracking(True)
    before = r.get_particles(0)
    cells = np.unique(before["cell"])[::7]
    pos = _mark(r, cells)
    r.step(1)
    t0 = r.get_tracked(0)
    r.pmerging("ti", [0.5])
    t1 = r.get_tracked(0)
    assert set(t1["trn"]) <= set(t0["trn"]) and 0 < t1["trn"].size < t0["trn"].size
    keep = np.isin(t0["trn"], t1["trn"])
    np.testing.assert_array_equal(t1["x"], t0["x"][keep])
    r.moving_window()
    t2 = r.get_tracked(0)
    on = t1["x"] >= 1.0  # layer 0 is erased by the window
    np.testing.assert_array_equal(t2["trn"], t1["trn"][on])
    np.testing.assert_array_equal(t2["x"], t1["x"][on] - 1)
    # particles loaded now are untracked
    r.add_particles(0, _photons(m=500, seed=4))
    assert r.get_tracked(0)["trn"].size == t2["trn"].size
    r.close()
