"""Parity of the CUDA path (through the C ABI) with the CPU checker.

FP64: bit-identical where the operation order is the reference's (fields
without particles, one particle, the first step of the particles, cell
indices and the traversal permutation); elsewhere within 1e-12 relative
(the current J is summed with atomics, so only its rounding order differs).
Mixed precision: within the tolerances stated per test.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests._cases import PUSHER_ID, SOLVER_ID, all_particles, small_case
from tests.conftest import gpu_available

pytestmark = pytest.mark.gpu

KIND = "ref" if O.available("ref", "parity") else "port"
FKEYS = ("ex", "ey", "ez", "bx", "by", "bz")
RTOL64 = 1e-12


def _gpu(case, species, precision="fp64"):
    from quill_b200.api import Region
    return Region(case.nx, case.ny, case.nz, case.dx, case.dx, case.dx, case.dt, species_cmr=species,
                  solver=case.solver, pusher=case.pusher, precision=precision)


def _cpu(case, icmr=()):
    return O.Region(case.nx, case.ny, case.nz, case.dx, case.dx, case.dx, case.dt,
                    solver=SOLVER_ID[case.solver], pusher=PUSHER_ID[case.pusher], icmr=icmr, kind=KIND)


def _load_both(case, fields, parts, species, precision="fp64"):
    icmr = tuple(c for c in species if c not in (-1.0, 1.0, 0.0))
    g, c = _gpu(case, species, precision), _cpu(case, icmr)
    for r in (g, c):
        r.set_fields(*[fields[k] for k in FKEYS])
        r.init_boundaries()
    for i, p in enumerate(parts):
        g.add_particles(i, p)
    if parts:
        c.add_particles(all_particles(parts))
    return g, c


def _rel(a, b):
    scale = np.max(np.abs(b))
    return 0.0 if scale == 0 else float(np.max(np.abs(a - b)) / scale)


def _split_by_species(cp, species):
    return [{k: v[cp["cmr"] == s] for k, v in cp.items()} for s in species]


@pytest.fixture(autouse=True)
def _need_gpu():
    if not gpu_available():
        pytest.skip("no CUDA device")


@pytest.mark.parametrize("solver", ["fdtd", "ndfx", "five_point"])
def test_fields_only_bitwise(solver):
    dtdx = 0.3 if solver == "five_point" else 0.5
    case, fields, _ = small_case(solver, dt_over_dx=dtdx, n=(23, 19, 17))
    g, c = _load_both(case, fields, [], (-1.0,))
    np.testing.assert_array_equal(g.get_fields(), c.get_fields())
    for _ in range(5):
        g.step(1)
        c.step(1)
    np.testing.assert_array_equal(g.get_fields(), c.get_fields())


@pytest.mark.parametrize("solver", ["fdtd", "ndfx", "five_point"])
@pytest.mark.parametrize("pusher", ["boris", "vay"])
def test_steps_fp64(solver, pusher):
    dtdx = 0.3 if solver == "five_point" else 0.5
    species = (-1.0, 1.0, 1 / 1836.15, 0.0)
    case, fields, parts = small_case(solver, pusher, dt_over_dx=dtdx, species=species, loaded_in_boundary=True)
    g, c = _load_both(case, fields, parts, species)
    for step in range(8):
        dg = g.step(1, external_bz=0.3)[0]
        dc = c.step(1, external_bz=0.3)[0]
        cp = _split_by_species(c.get_particles(), species)
        for si in range(len(species)):
            gp = g.get_particles(si)
            # cell indices and the traversal permutation are exact
            np.testing.assert_array_equal(gp["cell"], cp[si]["cell"], err_msg=f"step {step} species {si}")
            for k in ("x", "y", "z", "ux", "uy", "uz", "g", "q"):
                if step == 0:
                    np.testing.assert_array_equal(gp[k], cp[si][k], err_msg=f"step {step} {k}")
                else:
                    assert _rel(gp[k], cp[si][k]) <= RTOL64, (step, si, k, _rel(gp[k], cp[si][k]))
        fg, fc = g.get_fields(), c.get_fields()
        for a in range(12):
            assert _rel(fg[a], fc[a]) <= RTOL64, (step, a, _rel(fg[a], fc[a]))
        np.testing.assert_allclose(dg.as_array(), dc, rtol=1e-12, atol=0)


@pytest.mark.parametrize("crowd", [2, 3, 5, 9, 40, 150])
def test_rebin_front_orders_crowded_cell(crowd):
    """`crowd` particles from the 26 neighbours of one cell enter it in the
    same step, beside stayers: the front part of the cell's new list
    (arrivals in descending old traversal order, plist.cpp:22-39) goes
    through the pair exchange, the 4- and 8-entry networks, the insertion
    sort or the long-part kernel by its length.  Cell indices and order equal
    the reference's, and the positions are exact."""
    from tests._cases import small_case as _sc
    case, fields, _ = _sc("fdtd", "boris", n=(12, 12, 12))
    for k in fields:
        fields[k] = np.zeros_like(fields[k])
    rng = np.random.default_rng(crowd)
    T = np.array([6, 6, 6])
    offs = [np.array([a, b, c]) for a in (-1, 0, 1) for b in (-1, 0, 1) for c in (-1, 0, 1) if (a, b, c) != (0, 0, 0)]
    pos, u = [], []
    for m in range(crowd):
        dl = offs[m % 26]
        cell = T + dl
        frac = np.where(dl < 0, 0.93 + 0.05 * rng.random(3), np.where(dl > 0, 0.02 + 0.05 * rng.random(3),
                                                                       0.2 + 0.6 * rng.random(3)))
        pos.append(cell + frac)
        u.append(-0.3 * dl + np.where(dl == 0, 0.02 * rng.standard_normal(3), 0.0))
    for _ in range(3):  # stayers of the crowded cell
        pos.append(T + 0.3 + 0.4 * rng.random(3))
        u.append(0.01 * rng.standard_normal(3))
    pos, u = np.array(pos), np.array(u)
    cells = (pos[:, 0].astype(int) * case.ny + pos[:, 1].astype(int)) * case.nz + pos[:, 2].astype(int)
    o = np.argsort(cells, kind="stable")
    p = {"x": pos[o, 0], "y": pos[o, 1], "z": pos[o, 2], "ux": u[o, 0], "uy": u[o, 1], "uz": u[o, 2]}
    p["g"] = np.sqrt(1 + p["ux"] ** 2 + p["uy"] ** 2 + p["uz"] ** 2)
    p["q"] = -0.01 * (1 + 0.1 * rng.random(p["x"].size))
    p["cmr"] = np.full(p["x"].size, -1.0)
    g, c = _load_both(case, fields, [p], (-1.0,))
    Tc = (T[0] * case.ny + T[1]) * case.nz + T[2]
    for step in range(2):
        g.step(1)
        c.step(1)
        gp, cp = g.get_particles(0), c.get_particles()
        np.testing.assert_array_equal(gp["cell"], cp["cell"], err_msg=f"step {step}")
        for k in ("x", "y", "z"):
            # exact while the fields are the loaded zeros; then J's atomics
            # enter E (1e-12, as test_steps_fp64)
            if step == 0:
                np.testing.assert_array_equal(gp[k], cp[k], err_msg=f"step {step} {k}")
            else:
                assert _rel(gp[k], cp[k]) <= RTOL64, (step, k)
        # every particle sits in the crowded cell
        assert np.count_nonzero(gp["cell"] == Tc) == crowd + 3


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("waves", ["1", "0"])
@pytest.mark.parametrize("prefetch", ["1", "0"])
def test_push_chunks_per_block(monkeypatch, precision, waves, prefetch):
    """The pushes take block-sized chunks of the traversal, several per block
    when the grid is smaller than the particle count (QP_PUSH_WAVES = 1: one
    resident wave of blocks, here about ten chunks each) and one per block
    with QP_PUSH_WAVES = 0, with the next chunk's slot and cell loaded a
    chunk ahead (QP_PREFETCH = 1, the default) or not; the diagnostics summed
    per thread over its chunks and the particles equal the reference's (FP64
    to 1e-12; mixed to its tolerances)."""
    monkeypatch.setenv("QP_PUSH_WAVES", waves)
    monkeypatch.setenv("QP_PREFETCH", prefetch)
    species = (-1.0,)
    case, fields, parts = small_case("fdtd", "boris", n=(48, 48, 48), ppc=8, species=species)
    assert parts[0]["x"].size > 600000
    g, c = _load_both(case, fields, parts, species, precision=precision)
    for step in range(2):
        dg = g.step(1)[0]
        dc = c.step(1)[0]
    gp, cp = g.get_particles(0), c.get_particles()
    if precision == "fp64":
        np.testing.assert_array_equal(gp["cell"], cp["cell"])
        for k in ("x", "y", "z", "ux", "uy", "uz", "g"):
            assert _rel(gp[k], cp[k]) <= RTOL64, k
        # the diagnostics are sums over n particles (or cells) taken in
        # another order than the reference's loop: they agree to n x 2^-53
        n = max(gp["x"].size, case.nx * case.ny * case.nz)
        np.testing.assert_allclose(dg.as_array(), dc, rtol=n * 2.0 ** -53, atol=0)
    else:
        assert abs(gp["x"].size - cp["x"].size) <= max(2, gp["x"].size // 2000)
        np.testing.assert_allclose(dg.as_array(), dc, rtol=2e-5, atol=0)


def test_single_particle_bitwise():
    case, fields, parts = small_case("fdtd", "boris")
    p = {k: v[1000:1001] for k, v in parts[0].items()}
    p["ux"][:] = 2.0; p["uy"][:] = -1.5; p["uz"][:] = 1.2
    p["g"][:] = np.sqrt(1 + 4 + 2.25 + 1.44)
    g, c = _load_both(case, fields, [p], (-1.0,))
    for _ in range(10):
        g.step(1)
        c.step(1)
        np.testing.assert_array_equal(g.get_fields(), c.get_fields())
        gp, cp = g.get_particles(0), c.get_particles()
        for k in ("x", "y", "z", "ux", "uy", "uz", "g"):
            np.testing.assert_array_equal(gp[k], cp[k])


def test_empty_and_all_erased():
    case, fields, parts = small_case("fdtd", "boris")
    g, c = _load_both(case, fields, [], (-1.0, 1.0))
    d = g.step(3)
    assert g.count(0) == 0 and d[-1].N_qp_e == 0
    # particles only in the boundary layers: all erased on the first step
    p = {k: v[:4].copy() for k, v in parts[0].items()}
    p["x"][:] = [0.5, 0.7, case.nx - 1.5, case.nx - 0.2]
    g.add_particles(0, p)
    g.step(1)
    assert g.count(0) == 0


def test_checkpoint_restore_roundtrip():
    case, fields, parts = small_case("ndfx", "vay", species=(-1.0, 1 / 1836.15))
    g, _ = _load_both(case, fields, parts, (-1.0, 1 / 1836.15))
    g.step(2)
    g.checkpoint(1)
    g.step(3)
    f1, p1 = g.get_fields(), g.get_particles(0)
    g.restore(1)
    g.step(3)
    f2, p2 = g.get_fields(), g.get_particles(0)
    np.testing.assert_array_equal(p1["cell"], p2["cell"])
    for a in range(12):
        assert _rel(f2[a], f1[a]) <= RTOL64
    for k in ("x", "ux", "g"):
        assert _rel(p2[k], p1[k]) <= RTOL64


@pytest.mark.parametrize("solver", ["fdtd", "ndfx", "five_point"])
def test_mixed_precision_close(solver):
    """FP32 path against the FP64 checker: fields within 1e-4 of their peak
    after 5 steps, particle positions within 1e-4 cells."""
    dtdx = 0.3 if solver == "five_point" else 0.5
    species = (-1.0, 1 / 1836.15)
    case, fields, parts = small_case(solver, "boris", dt_over_dx=dtdx, species=species)
    g, c = _load_both(case, fields, parts, species, precision="mixed")
    for _ in range(5):
        g.step(1)
        c.step(1)
    fg, fc = g.get_fields(), c.get_fields()
    for a in range(6):
        assert _rel(fg[a], fc[a]) <= 1e-4, (a, _rel(fg[a], fc[a]))
    cp = _split_by_species(c.get_particles(), species)
    gp = g.get_particles(0)
    if gp["x"].size == cp[0]["x"].size and np.array_equal(gp["cell"], cp[0]["cell"]):
        assert np.max(np.abs(gp["x"] - cp[0]["x"])) < 1e-4
    else:
        # a particle within FP32 round-off of a face may land in the
        # neighbouring cell; counts must still agree closely
        assert abs(gp["x"].size - cp[0]["x"].size) <= max(2, gp["x"].size // 2000)


def test_moving_window_fp64():
    """spatial_region::moving_window (advance.cpp:389-454) on the GPU: exact
    data movement (bit-identical right after loading), then steps and
    shifts alternating stay within the step parity tolerance."""
    species = (-1.0, 1 / 1836.15)
    case, fields, parts = small_case("fdtd", "boris", species=species)
    g, c = _load_both(case, fields, parts, species)
    g.moving_window()
    c.moving_window()
    assert np.array_equal(g.get_fields()[[0, 1, 2, 3, 4, 5, 9, 10, 11]], c.get_fields()[[0, 1, 2, 3, 4, 5, 9, 10, 11]])
    cp = _split_by_species(c.get_particles(), species)
    for i in range(len(species)):
        gp = g.get_particles(i)
        for k in ("x", "y", "z", "ux", "q", "cell"):
            assert np.array_equal(gp[k], cp[i][k]), (i, k)
    for _ in range(3):
        g.step(1)
        c.step(1)
        g.moving_window()
        c.moving_window()
        fg, fc = g.get_fields(), c.get_fields()
        for a in range(12):
            assert _rel(fg[a], fc[a]) <= RTOL64, a
        cp = _split_by_species(c.get_particles(), species)
        for i in range(len(species)):
            gp = g.get_particles(i)
            assert np.array_equal(gp["cell"], cp[i]["cell"])
            for k in ("x", "ux", "q"):
                assert _rel(gp[k], cp[i][k]) <= RTOL64


def test_moving_window_mixed():
    species = (-1.0,)
    case, fields, parts = small_case("fdtd", "boris", species=species)
    g, c = _load_both(case, fields, parts, species, precision="mixed")
    for _ in range(3):
        g.step(1)
        c.step(1)
        g.moving_window()
        c.moving_window()
    fg, fc = g.get_fields(), c.get_fields()
    for a in range(6):
        assert _rel(fg[a], fc[a]) <= 1e-4, a
    assert abs(g.count(0) - c.count()) <= max(2, c.count() // 2000)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_field_slices_and_max_w(precision):
    """qp_dump_field_slices gives the output writers' lines and plane of every
    field plane (fout.cpp:180-235); qp_max_w the max of E^2 + B^2 over an x
    range (get_max_w, low-level.cpp:512-532)."""
    species = (-1.0,)
    case, fields, parts = small_case("fdtd", "boris", species=species)
    g, _ = _load_both(case, fields, parts, species, precision)
    g.step(2)
    f = g.get_fields()
    nx, ny, nz = case.nx, case.ny, case.nz
    ix = nx // 2 + 1
    s = g.field_slices(ix)
    for a in range(12):
        want = np.concatenate([np.concatenate([f[a, i, :, nz // 2], f[a, i, ny // 2, :]]) for i in range(nx)] +
                              [f[a, ix].reshape(-1)])
        np.testing.assert_array_equal(s[a], want)
    w = (f[:6] ** 2).sum(0)
    for i0, i1 in ((0, nx), (nx - 6, nx - 4), (3, 4)):
        np.testing.assert_allclose(g.max_w(i0, i1), w[i0:i1].max(), rtol=1e-12 if precision == "fp64" else 1e-6)
    assert g.max_w(5, 5) == 0.0
