"""Energy carried off by erased particles (qp_set_erased_tracking): with it,
the region's energy balance closes.

* Photons move ballistically with constant energy g q, so the photon energy
  left in the region plus the energy of the photons erased so far equals the
  initial photon energy to round-off, whichever boundary they cross.
* Electrons loaded in the p_boundary layers are erased before their first
  push with their loaded energy: the erased energy of that step is
  -b sum (g - 1) q, with compute_energy's normalisation b (main.cpp:2327).
"""
import math

import numpy as np
import pytest

from tests.conftest import gpu_available

pytestmark = pytest.mark.gpu

N = (20, 18, 16)
DX = 2 * math.pi / 16
DT = 0.5 * DX


def _b(lambda_cm=1e-4):
    return 8.2e-14 * DX ** 3 * 1.11485e13 * lambda_cm / (8 * math.pi ** 3)


def _sorted(parts):
    cells = (parts["x"].astype(int) * N[1] + parts["y"].astype(int)) * N[2] + parts["z"].astype(int)
    o = np.argsort(cells, kind="stable")
    return {k: v[o] for k, v in parts.items()}


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_photon_energy_balance_closes(precision):
    if not gpu_available():
        pytest.skip("needs a CUDA device")
    from quill_b200.api import Region
    rng = np.random.default_rng(3)
    m = 4000
    u = rng.standard_normal((3, m)) * 5.0
    g = np.sqrt((u * u).sum(0))
    parts = _sorted({"x": rng.uniform(1, N[0] - 3, m), "y": rng.uniform(1, N[1] - 3, m),
                     "z": rng.uniform(1, N[2] - 3, m), "ux": u[0], "uy": u[1], "uz": u[2], "g": g,
                     "q": rng.uniform(0.01, 0.1, m)})
    r = Region(*N, DX, DX, DX, DT, species_cmr=(0.0,), precision=precision)
    r.set_fields(*np.zeros((6,) + N))
    r.init_boundaries()
    r.add_particles(0, parts)
    r.set_erased_tracking(True)
    w0 = _b() * float(np.sum(parts["g"] * parts["q"]))
    d = r.step(24)
    lost = np.cumsum([x.energy_erased for x in d])
    left = np.array([x.energy_ph for x in d])
    r.close()
    assert d[-1].n_macro[0] < m // 2          # most photons left the region
    tol = 1e-12 if precision == "fp64" else 1e-6
    np.testing.assert_allclose(left + lost, w0, rtol=tol)


def test_electrons_in_boundary_layers_erased_with_their_energy():
    if not gpu_available():
        pytest.skip("needs a CUDA device")
    from quill_b200.api import Region
    rng = np.random.default_rng(4)
    m = 300
    # positions in the layers p_boundary erases: 0, n-2, n-1 on one axis each
    x = rng.uniform(2, N[0] - 3, m)
    y = rng.uniform(2, N[1] - 3, m)
    z = rng.uniform(2, N[2] - 3, m)
    which = rng.integers(0, 3, m)
    x[which == 0] = rng.choice([0.5, N[0] - 1.5, N[0] - 0.5], (which == 0).sum())
    y[which == 1] = rng.choice([0.5, N[1] - 1.5, N[1] - 0.5], (which == 1).sum())
    z[which == 2] = rng.choice([0.5, N[2] - 1.5, N[2] - 0.5], (which == 2).sum())
    u = rng.standard_normal((3, m))
    g = np.sqrt(1 + (u * u).sum(0))
    q = -rng.uniform(0.01, 0.1, m)
    parts = _sorted({"x": x, "y": y, "z": z, "ux": u[0], "uy": u[1], "uz": u[2], "g": g, "q": q})
    r = Region(*N, DX, DX, DX, DT)
    r.set_fields(*np.zeros((6,) + N))
    r.init_boundaries()
    r.add_particles(0, parts)
    r.set_erased_tracking(True)
    d = r.step(1)[0]
    r.close()
    assert d.n_macro[0] == 0
    want = -_b() * float(np.sum((parts["g"] - 1) * parts["q"]))
    assert abs(d.energy_erased - want) <= 1e-12 * abs(want)


def test_tracking_off_reports_zero():
    if not gpu_available():
        pytest.skip("needs a CUDA device")
    from quill_b200.api import Region
    r = Region(*N, DX, DX, DX, DT)
    r.set_fields(*np.zeros((6,) + N))
    r.init_boundaries()
    r.add_particles(0, {"x": np.array([0.5]), "y": np.array([5.5]), "z": np.array([5.5]), "ux": np.zeros(1),
                        "uy": np.zeros(1), "uz": np.zeros(1), "g": np.ones(1) * 2, "q": -np.ones(1)})
    d = r.step(1)[0]
    r.close()
    assert d.energy_erased == 0.0 and d.n_macro[0] == 0


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_catching_records_every_erased_photon(precision):
    """Catching (delete_particle with catching_enabled, low-level.cpp:247-259):
    one record per erased particle, outside the region, carrying the energy
    the erased-energy sum counted."""
    if not gpu_available():
        pytest.skip("needs a CUDA device")
    from quill_b200.api import Region
    rng = np.random.default_rng(5)
    m = 3000
    u = rng.standard_normal((3, m)) * 5.0
    parts = _sorted({"x": rng.uniform(1, N[0] - 3, m), "y": rng.uniform(1, N[1] - 3, m),
                     "z": rng.uniform(1, N[2] - 3, m), "ux": u[0], "uy": u[1], "uz": u[2],
                     "g": np.sqrt((u * u).sum(0)), "q": rng.uniform(0.01, 0.1, m)})
    r = Region(*N, DX, DX, DX, DT, species_cmr=(0.0,), precision=precision)
    r.set_fields(*np.zeros((6,) + N))
    r.init_boundaries()
    r.add_particles(0, parts)
    r.set_erased_tracking(True)
    r.set_catching(True, capacity=m)
    d = r.step(24)
    c = r.get_caught()
    again = r.get_caught()
    n_end = r.count(0)
    r.close()
    assert c["dropped"] == 0 and again["x"].size == 0
    assert c["x"].size == m - n_end and np.all(c["species"] == 0)
    i, j, k = (np.floor(c[a]).astype(int) for a in ("x", "y", "z"))
    inside = (i > 0) & (i < N[0] - 2) & (j > 0) & (j < N[1] - 2) & (k > 0) & (k < N[2] - 2)
    assert not inside.any()
    tol = 1e-12 if precision == "fp64" else 1e-6
    np.testing.assert_allclose(_b() * np.sum(c["g"] * c["q"]), sum(x.energy_erased for x in d), rtol=tol)
    np.testing.assert_allclose(sum(x.energy_erased_sp[0] for x in d), sum(x.energy_erased for x in d), rtol=1e-14)


def test_catching_capacity_overflow_is_counted():
    if not gpu_available():
        pytest.skip("needs a CUDA device")
    from quill_b200.api import Region
    m = 300
    x = np.full(m, 0.5)  # all in the layer p_boundary erases
    parts = {"x": x, "y": np.linspace(2.1, 12.9, m), "z": np.full(m, 5.5), "ux": np.zeros(m), "uy": np.zeros(m),
             "uz": np.zeros(m), "g": np.ones(m) * 1.5, "q": -np.ones(m) * 0.01}
    r = Region(*N, DX, DX, DX, DT)
    r.set_fields(*np.zeros((6,) + N))
    r.init_boundaries()
    r.add_particles(0, _sorted(parts))
    r.set_catching(True, capacity=100)
    r.step(1)
    c = r.get_caught()
    r.close()
    assert c["x"].size == 100 and c["dropped"] == m - 100


def _qed_region(precision, with_photons):
    """Electrons across a strong Bz (chi ~ 1) and, optionally, energetic
    photons for pair creation, in the middle of a 16^3 box."""
    from quill_b200.api import Region
    from tests import test_qed as Q
    fields, e, ph = Q._emission_case(0)
    r = Region(Q.N, Q.N, Q.N, Q.DX, Q.DX, Q.DX, Q.DT, species_cmr=(-1.0, 1.0, 0.0), solver="fdtd", pusher="boris",
               qed=True, seed=11, precision=precision)
    r.set_fields(*[fields[k] for k in ("ex", "ey", "ez", "bx", "by", "bz")])
    r.init_boundaries()
    if with_photons:
        r.add_particles(2, Q._sort(ph))
    else:
        r.add_particles(0, Q._sort(e))
    return r


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_dump_photons_records_every_emitted_photon(precision):
    """dump_photons (advance.cpp:302-306): the photons the electrons emit are
    deleted as they are born; each is recorded with its energy, which is the
    photon species' erased energy; the photon species stays empty."""
    if not gpu_available():
        pytest.skip("needs a CUDA device")
    r = _qed_region(precision, with_photons=False)
    r.set_dump_photons(True)
    total = 0.0
    n_rec = 0
    for _ in range(3):
        d = r.step(1)[0]
        c = r.get_caught()
        assert np.all(c["species"] == 2)
        n_rec += c["x"].size
        assert d.energy_erased_sp[2] == pytest.approx(np.sum(c["g"] * c["q"]) * _b(), rel=1e-12, abs=0)
        total += d.energy_erased_sp[2]
    assert r.count(2) == 0 and n_rec > 100 and total > 0
    assert r.count(0) > 0
    r.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_pair_creation_is_not_an_erasure(precision):
    """A photon that becomes a pair is deleted without a record
    (delete_particle without force_delete inside the box): with catching on,
    photons in the middle of the box make pairs and nothing is recorded."""
    if not gpu_available():
        pytest.skip("needs a CUDA device")
    r = _qed_region(precision, with_photons=True)
    r.set_erased_tracking(True)
    r.set_catching(True)
    n0 = r.count(2)
    d = r.step(1)[0]
    assert r.count(0) > 0 and r.count(2) < n0    # pairs were made
    c = r.get_caught()
    assert c["x"].size == 0 and d.energy_erased == 0.0
    r.close()
