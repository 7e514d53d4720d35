"""QED: device rate functions against the reference's (mc.cpp:26-116), the
counter-based random numbers against the published Philox4x32-10 answers,
and photon-emission / pair-creation statistics of whole steps against the
reference run with 16 seeds (agreement within 3 sigma): photon, electron
and positron counts and energies, and their energy spectra bin by bin with
the reference's spectrum normalisation."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.conftest import gpu_available

KIND = "ref" if O.available("ref", "parity") else "port"


def _rate_samples(n, seed=5):
    rng = np.random.default_rng(seed)
    e = rng.standard_normal((n, 3)) * 10 ** rng.uniform(1, 5, (n, 1))
    b = rng.standard_normal((n, 3)) * 10 ** rng.uniform(1, 5, (n, 1))
    u = rng.standard_normal((n, 3)) * 10 ** rng.uniform(0, 3.5, (n, 1))
    g = np.sqrt(1 + (u * u).sum(1))
    r = rng.uniform(0, 1, n)
    chi = 10 ** rng.uniform(-3, 1, n)
    return np.column_stack([e, b, u, g, r, chi])


@pytest.mark.gpu
def test_device_rates_match_reference():
    if not gpu_available():
        pytest.skip("no CUDA device")
    from quill_b200.api import eval_qed_rates
    smp = _rate_samples(4000)
    out = eval_qed_rates(smp)
    reg = O.Region(8, 8, 8, 0.4, 0.4, 0.4, 0.2, kind=KIND)
    for row, o in zip(smp, out):
        e, b, u, g, r, chi = row[0:3], row[3:6], row[6:9], row[9], row[10], row[11]
        ref_chi = reg.chi(e, b, u, g)
        ref_w, ref_r = reg.w(g, r, chi)
        ref_tw = reg.tilde_w(g, r, chi)
        ref_W = reg.mathcal_W(e, b)
        # CUDA's pow/exp/tanh are within a few ulp of the host libm: allow
        # 1e-12 relative (the rates contain a difference of two terms)
        np.testing.assert_allclose(o[0], ref_chi, rtol=1e-13)
        np.testing.assert_allclose(o[2], ref_r, rtol=1e-15)
        np.testing.assert_allclose(o[1], ref_w, rtol=1e-11, atol=1e-300)
        np.testing.assert_allclose(o[3], ref_tw, rtol=1e-11, atol=1e-300)
        np.testing.assert_allclose(o[4], ref_W, rtol=1e-11, atol=1e-300)


# ---------------------------------------------------------------------------
# whole-step statistics
# ---------------------------------------------------------------------------
N = 16
DX = 2 * np.pi / 16
DT = 0.5 * DX
B0 = 400.0       # uniform Bz, chi ~ 1 for gamma ~ 1e3
GAMMA0 = 1000.0
STEPS = 6


def _emission_case(seed, n_e=4000, n_ph=4000):
    rng = np.random.default_rng(seed)
    fields = {k: np.zeros((N, N, N)) for k in ("ex", "ey", "ez", "bx", "by", "bz")}
    fields["bz"][:] = B0
    parts = []
    # electrons moving along +y (perpendicular to B), starting in x in [2, 6)
    x = rng.uniform(2, 6, n_e); y = rng.uniform(2, 5, n_e); z = rng.uniform(2, 13, n_e)
    u = np.sqrt(GAMMA0 ** 2 - 1)
    e = {"x": x, "y": y, "z": z, "ux": np.zeros(n_e), "uy": np.full(n_e, u), "uz": np.zeros(n_e),
         "g": np.full(n_e, GAMMA0), "q": np.full(n_e, -1e-8), "cmr": np.full(n_e, -1.0)}
    # photons for pair creation: gamma 4000 along +y
    xp = rng.uniform(8, 12, n_ph); yp = rng.uniform(2, 5, n_ph); zp = rng.uniform(2, 13, n_ph)
    ph = {"x": xp, "y": yp, "z": zp, "ux": np.zeros(n_ph), "uy": np.full(n_ph, 4000.0), "uz": np.zeros(n_ph),
          "g": np.full(n_ph, 4000.0), "q": np.full(n_ph, 1e-8), "cmr": np.zeros(n_ph)}
    return fields, e, ph


def _sort(p):
    cell = (p["x"].astype(int) * N + p["y"].astype(int)) * N + p["z"].astype(int)
    o = np.argsort(cell, kind="stable")
    return {k: v[o] for k, v in p.items()}


# energy bins of the spectra, as write_spectrum_phasespace bins them
# (main.cpp:535-600): photons by g * 0.511 / deps_ph, leptons by
# (g - 1) * 0.511 / deps, weight q (its magnitude), normalised to dN/deps in
# 1/MeV with the reference's factor (main.cpp:683-700)
DEPS_PH, NEPS_PH = 100.0, 24      # MeV: the 2.04 GeV pair photons and the emitted ones below 511 MeV
DEPS_L, NEPS_L = 100.0, 24        # MeV: electrons from 511 MeV down, pairs up to 2 GeV
LAMBDA_CM = 1e-4
SPEC_NORM = 1.11485e13 * LAMBDA_CM * DX * DX * DX / (8 * np.pi ** 3)


def _spectrum(p, photon, deps, neps):
    e = (p["g"] if photon else p["g"] - 1) * 0.511 / deps
    i = e.astype(int)
    keep = (i > -1) & (i < neps)
    return np.bincount(i[keep], weights=np.abs(p["q"][keep]), minlength=neps) * SPEC_NORM / deps


def _stats_from(parts_e, parts_p, parts_ph):
    return {"n_ph": parts_ph["x"].size, "e_ph": parts_ph["g"].sum(), "n_p": parts_p["x"].size,
            "e_e": parts_e["g"].sum(),
            "spec_ph": _spectrum(parts_ph, True, DEPS_PH, NEPS_PH),
            "spec_e": _spectrum(parts_e, False, DEPS_L, NEPS_L),
            "spec_p": _spectrum(parts_p, False, DEPS_L, NEPS_L)}


def _ref_stats(seed):
    fields, e, ph = _emission_case(0)
    reg = O.Region(N, N, N, DX, DX, DX, DT, solver=0, pusher=1, qed=True, seed=seed, kind=KIND)
    reg.set_fields(*[fields[k] for k in ("ex", "ey", "ez", "bx", "by", "bz")])
    reg.init_boundaries()
    allp = _sort({k: np.concatenate([e[k], ph[k]]) for k in e})
    reg.add_particles(allp)
    reg.step(STEPS)
    p = reg.get_particles()
    sel = lambda c: {k: v[p["cmr"] == c] for k, v in p.items()}
    return _stats_from(sel(-1.0), sel(1.0), sel(0.0))


_REF_CACHE = {}


def _ref_stats_cached(seed):
    if seed not in _REF_CACHE:
        _REF_CACHE[seed] = _ref_stats(seed)
    return _REF_CACHE[seed]


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_qed_step_statistics_vs_reference(precision):
    """Emission, recoil and pair creation; the mixed path evaluates the
    rates in FP32 against the same per-step rejection."""
    if not gpu_available():
        pytest.skip("no CUDA device")
    if KIND != "ref":
        pytest.skip("whole-step QED statistics need the compiled reference")
    from quill_b200.api import Region
    ref = [_ref_stats_cached(1 + s) for s in range(16)]
    gpu = []
    for seed in range(16):
        fields, e, ph = _emission_case(0)
        g = Region(N, N, N, DX, DX, DX, DT, species_cmr=(-1.0, 1.0, 0.0), solver="fdtd", pusher="boris",
                   qed=True, seed=1000 + seed, precision=precision)
        g.set_fields(*[fields[k] for k in ("ex", "ey", "ez", "bx", "by", "bz")])
        g.init_boundaries()
        g.add_particles(0, _sort(e))
        g.add_particles(2, _sort(ph))
        g.step(STEPS)
        gpu.append(_stats_from(g.get_particles(0), g.get_particles(1), g.get_particles(2)))
        g.close()
    for key in ("n_ph", "e_ph", "n_p", "e_e"):
        r = np.array([x[key] for x in ref], dtype=float)
        v = np.array([x[key] for x in gpu], dtype=float)
        # difference of the two 16-seed means within 3 sigma of that difference
        sig = np.sqrt(r.var(ddof=1) / r.size + v.var(ddof=1) / v.size)
        assert abs(v.mean() - r.mean()) <= 3 * sig + 1e-12 * abs(r.mean()), (key, v.mean(), r.mean(), sig)
        assert r.mean() > 0
    # spectra, bin by bin (photons, electrons, positrons): the difference of
    # the 16-seed means within 3 sigma of that difference; with about 70
    # populated bins tested at 3 sigma, one exceedance is allowed (its
    # expected number by chance is about 0.2), none beyond 4 sigma.  Bins that
    # are empty in both runs are skipped.
    over3 = []
    tested = 0
    for key in ("spec_ph", "spec_e", "spec_p"):
        r = np.array([x[key] for x in ref])
        v = np.array([x[key] for x in gpu])
        assert r.sum() > 0, key
        for b in range(r.shape[1]):
            if not (r[:, b].any() or v[:, b].any()):
                continue
            tested += 1
            sig = np.sqrt(r[:, b].var(ddof=1) / r.shape[0] + v[:, b].var(ddof=1) / v.shape[0])
            dev = abs(v[:, b].mean() - r[:, b].mean())
            assert dev <= 4 * sig + 1e-12 * abs(r[:, b].mean()), (key, b, v[:, b].mean(), r[:, b].mean(), sig)
            if dev > 3 * sig + 1e-12 * abs(r[:, b].mean()):
                over3.append((key, b))
    assert tested >= 20
    assert len(over3) <= 1, over3


# Schwinger pairs from a uniform Ex of 0.073 e_s: about 1e-2 pairs per
# interior cell and step, so a 16^3 box makes about 17 per step
E_VAC = 0.073 * 1e-4 / 2.4263086e-10


def _vacuum_counts_ref(seed, steps=2):
    reg = O.Region(N, N, N, DX, DX, DX, DT, solver=0, pusher=1, qed=True, seed=seed, kind=KIND)
    z = np.zeros((N, N, N))
    reg.set_fields(np.full((N, N, N), E_VAC), z, z, z, z, z)
    reg.init_boundaries()
    out = []
    for _ in range(steps):
        reg.step(1)
        p = reg.get_particles()
        out.append(((p["cmr"] == -1).sum(), (p["cmr"] == 1).sum()))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_vacuum_pairs_vs_reference(precision):
    if not gpu_available():
        pytest.skip("no CUDA device")
    if KIND != "ref":
        pytest.skip("vacuum pair statistics need the compiled reference")
    from quill_b200.api import Region
    ref = np.array([_vacuum_counts_ref(1 + s) for s in range(16)], dtype=float)
    gpu = []
    z = np.zeros((N, N, N))
    for seed in range(16):
        g = Region(N, N, N, DX, DX, DX, DT, species_cmr=(-1.0, 1.0, 0.0), solver="fdtd", pusher="boris",
                   qed=True, seed=500 + seed, precision=precision)
        g.set_fields(np.full((N, N, N), E_VAC), z, z, z, z, z)
        g.init_boundaries()
        rows = []
        for _ in range(2):
            g.step(1)
            rows.append((g.count(0), g.count(1)))
        gpu.append(rows)
        g.close()
    gpu = np.array(gpu, dtype=float)
    assert ref[:, 0, 0].mean() > 3
    # step 1: the pairs themselves; step 2 adds the cascade they start (the
    # field accelerates them to chi ~ 1e2 within a step)
    for step in range(2):
        for sp in range(2):
            r, v = ref[:, step, sp], gpu[:, step, sp]
            sig = np.sqrt(r.var(ddof=1) / r.size + v.var(ddof=1) / v.size)
            assert abs(v.mean() - r.mean()) <= 3 * sig, (step, sp, v.mean(), r.mean(), sig)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_resting_leptons_do_not_emit(precision):
    """A lepton at rest (g = 1) cannot emit: w's range check (1 - r) g >= 1
    rejects every draw (mc.cpp:40-74).  In FP32, 1 - r rounds to 1 for draws
    below 2^-24, so the mixed path takes the check on the FP64 draw; without
    it a resting electron in a strong field emitted a photon along an
    undefined direction (NaN).  Cold electrons in a field of 1500 m c omega /
    e over 2 steps: no NaN, and no photon from the first step."""
    if not gpu_available():
        pytest.skip("no CUDA device")
    from quill_b200.api import Region
    n = 16
    rng = np.random.default_rng(3)
    m = 200000
    p = {"x": rng.uniform(3, 12, m), "y": rng.uniform(3, 12, m), "z": rng.uniform(3, 12, m),
         "ux": np.zeros(m), "uy": np.zeros(m), "uz": np.zeros(m), "g": np.ones(m), "q": np.full(m, -1e-3)}
    z = np.zeros((n, n, n))
    g = Region(n, n, n, DX, DX, DX, DT, species_cmr=(-1.0, 1.0, 0.0), solver="fdtd", pusher="vay", qed=True,
               seed=7, precision=precision)
    g.set_fields(z, np.full((n, n, n), 1500.0), z, z, z, np.full((n, n, n), 1500.0))
    g.init_boundaries()
    g.add_particles(0, _sort(p))
    g.step(1)
    assert g.count(2) == 0
    g.step(1)  # the electrons now move; emission may start, but nothing is NaN
    for s in range(3):
        q = g.get_particles(s)
        for k in ("x", "ux", "g"):
            assert np.isfinite(q[k]).all(), (s, k)
