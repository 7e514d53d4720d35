"""Particle merging on the GPU (qp_pmerging) against the reference's
spatial_region::pmerging (mc.cpp:198-462).

The reference draws its deletions from one sequential random stream, the GPU
from a counter-based one, so the deleted particles are compared in
distribution: the number deleted per species against its binomial (or
Poisson-binomial, "nl") expectation and against the reference's own count,
within 5 sigma.  Everything else is exact: the survivors keep their order,
cells and states; their weights are rescaled by the reference's factors;
each species keeps its total charge; and the merged state then steps like
the checker loaded with the same particles (1e-12 relative, FP64).
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests._cases import all_particles, small_case
from tests.conftest import gpu_available

pytestmark = pytest.mark.gpu

KIND = "ref" if O.available("ref", "parity") else "port"
SPECIES = (-1.0, 1.0, 0.0, 1 / 1836.15)
FKEYS = ("ex", "ey", "ez", "bx", "by", "bz")


def _case(seed=5):
    case, fields, parts = small_case(species=SPECIES, ppc=4, seed=seed)
    rng = np.random.default_rng(seed + 20)
    for p in parts:
        p["q"] = p["q"] * rng.uniform(0.3, 3.0, p["q"].size)
    return case, fields, parts


def _gpu(case, fields, parts, precision="fp64"):
    from quill_b200.api import Region
    r = Region(case.nx, case.ny, case.nz, case.dx, case.dx, case.dx, case.dt, species_cmr=SPECIES,
               solver=case.solver, pusher=case.pusher, precision=precision, seed=17)
    r.set_fields(*[fields[k] for k in FKEYS])
    r.init_boundaries()
    for i, p in enumerate(parts):
        r.add_particles(i, {k: v for k, v in p.items() if k != "cmr"})
    return r


def _subsequence(before, after):
    """Indices of `after`'s particles in `before` (same cell and position),
    checking that they appear in the same order."""
    key_b = list(zip(before["cell"], before["x"], before["y"], before["z"]))
    idx, j = [], 0
    for key in zip(after["cell"], after["x"], after["y"], after["z"]):
        while key_b[j] != key:
            j += 1
        idx.append(j)
        j += 1
    return np.array(idx, dtype=np.int64)


def _sgn(i):
    return -1.0 if SPECIES[i] == -1 else 1.0


def _ppd(q, q0):
    return 1.0 / (1.0 + (2.0 * q / q0) ** 4)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_ti_deletion_rescale_and_order(precision):
    if not gpu_available():
        pytest.skip("needs a CUDA device")
    case, fields, parts = _case()
    r = _gpu(case, fields, parts, precision)
    r.step(1)
    before = [r.get_particles(i) for i in range(len(SPECIES))]
    ppd = 0.3
    r.pmerging("ti", [ppd])
    after = [r.get_particles(i) for i in range(len(SPECIES))]
    rtol = 1e-12 if precision == "fp64" else 1e-6
    for i, (b, a) in enumerate(zip(before, after)):
        n = b["x"].size
        dele = n - a["x"].size
        assert abs(dele - ppd * n) <= 5 * np.sqrt(n * ppd * (1 - ppd)) + 1, (i, dele, n)
        idx = _subsequence(b, a)
        for k in ("ux", "uy", "uz", "g"):
            np.testing.assert_array_equal(a[k], b[k][idx])
        # one factor for the species: a / (a - deleted charge); charge kept
        ratio = a["q"] / b["q"][idx]
        np.testing.assert_allclose(ratio, ratio[0], rtol=rtol)
        np.testing.assert_allclose(a["q"].sum(), b["q"].sum(), rtol=rtol)
    r.close()


def test_nl_prefers_light_particles_and_keeps_charge():
    if not gpu_available():
        pytest.skip("needs a CUDA device")
    case, fields, parts = _case(seed=6)
    r = _gpu(case, fields, parts)
    before = [r.get_particles(i) for i in range(len(SPECIES))]
    ppd = [0.6, 0.4, 0.8, 0.5]
    r.pmerging("nl", ppd)
    after = [r.get_particles(i) for i in range(len(SPECIES))]
    for i, (b, a) in enumerate(zip(before, after)):
        s = _sgn(i)
        qabs = s * b["q"]
        pdel = ppd[i] * _ppd(qabs, qabs.sum() / qabs.size)
        mean, var = pdel.sum(), (pdel * (1 - pdel)).sum()
        dele = b["x"].size - a["x"].size
        assert abs(dele - mean) <= 5 * np.sqrt(var) + 1, (i, dele, mean)
        idx = _subsequence(b, a)
        # survivors: q / (1 - pdel(q)), then one factor for the species
        ratio = a["q"] / (b["q"][idx] / (1 - pdel[idx]))
        np.testing.assert_allclose(ratio, ratio[0], rtol=1e-12)
        np.testing.assert_allclose(a["q"].sum(), b["q"].sum(), rtol=1e-12)
        # light particles are deleted more often than heavy ones
        light = qabs < np.median(qabs)
        kept = np.zeros(b["x"].size, bool)
        kept[idx] = True
        assert (~kept[light]).mean() > (~kept[~light]).mean()
    r.close()


@pytest.mark.parametrize("mode,ppd", [("ti", [0.3]), ("nl", [0.6, 0.4, 0.8, 0.5])])
def test_deleted_counts_agree_with_reference(mode, ppd):
    if not gpu_available():
        pytest.skip("needs a CUDA device")
    case, fields, parts = _case(seed=7)
    r = _gpu(case, fields, parts)
    n0 = [r.count(i) for i in range(len(SPECIES))]
    r.pmerging(mode, ppd)
    ng = [r.count(i) for i in range(len(SPECIES))]
    r.close()
    ref = O.Region(case.nx, case.ny, case.nz, case.dx, case.dx, case.dx, case.dt, solver=0, pusher=1,
                   icmr=(1 / 1836.15,), kind=KIND)
    ref.set_fields(*[fields[k] for k in FKEYS])
    ref.init_boundaries()
    ref.add_particles(all_particles(parts))
    ref.pmerging(mode, ppd)
    pc = ref.get_particles()
    for i, c in enumerate(SPECIES):
        nr = int(np.sum(pc["cmr"] == c))
        p = (n0[i] - ng[i]) / n0[i]
        sigma = np.sqrt(2 * n0[i] * max(p * (1 - p), 1e-3))
        assert abs(ng[i] - nr) <= 5 * sigma + 1, (i, ng[i], nr)


def test_merged_state_steps_like_the_checker():
    if not gpu_available():
        pytest.skip("needs a CUDA device")
    case, fields, parts = _case(seed=8)
    r = _gpu(case, fields, parts)
    r.pmerging("ti", [0.25])
    f = r.get_fields()
    merged = [r.get_particles(i) for i in range(len(SPECIES))]
    ref = O.Region(case.nx, case.ny, case.nz, case.dx, case.dx, case.dx, case.dt, solver=0, pusher=1,
                   icmr=(1 / 1836.15,), kind=KIND)
    ref.set_fields(*f[:6])
    ref.init_boundaries()
    cat = {k: np.concatenate([m[k] for m in merged]) for k in ("x", "y", "z", "ux", "uy", "uz", "g", "q")}
    cat["cmr"] = np.concatenate([np.full(m["x"].size, c) for m, c in zip(merged, SPECIES)])
    cells = np.concatenate([m["cell"] for m in merged])
    o = np.argsort(cells, kind="stable")
    ref.add_particles({k: v[o] for k, v in cat.items()})
    r.step(2)
    ref.step(2)
    fg, fr = r.get_fields(), ref.get_fields()
    for a in range(9):
        scale = max(np.abs(fr[a]).max(), 1e-300)
        assert np.abs(fg[a] - fr[a]).max() <= 1e-12 * scale + 1e-300, a
    r.close()


def test_bad_arguments():
    if not gpu_available():
        pytest.skip("needs a CUDA device")
    from quill_b200.api import QPError
    case, fields, parts = _case()
    r = _gpu(case, fields, parts)
    with pytest.raises(QPError):
        r.pmerging("ti", [1.0])
    with pytest.raises(QPError):
        r.pmerging("nl", [0.1, -0.2, 0.1, 0.1])
    r.close()
