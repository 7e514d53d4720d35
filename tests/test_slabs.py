"""A box cut into overlapping x-slab regions (the reference's n_sr > 1 runs,
main.cpp:1286-1514, 2155-2184, balancing.cpp).

CPU: the load-balancing arithmetic against the reference's own
balancing.cpp; slab runs of the restatement against slab runs of the
reference's spatial_region bit for bit (the exchange moves particles between
frames with a floating-point add, so a slab run and a one-region run agree
to rounding only, which is checked too); the exchange over torch.distributed
with gloo ranks against the in-process exchange, bit for bit.

GPU: library regions on one GPU, exchanging host or device buffers, against
the restatement's slab run (FP64: 1e-12, J is summed by atomics)."""
import os
import socket
import subprocess
import tempfile

import numpy as np
import pytest

from oracle import oracle as O
from quill_b200 import slabs as S
from tests._cases import PUSHER_ID, SOLVER_ID, all_particles, small_case
from tests.conftest import gpu_available

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FIELD_PLANES = ("ex", "ey", "ez", "bx", "by", "bz")

needs_ref = pytest.mark.skipif(not O.available("ref", "parity"),
                               reason="reference not compiled here (make -C oracle ref)")


def _ensure_port():
    if not O.available("port", "parity"):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True, capture_output=True)


def _case(solver="fdtd", pusher="boris", nx=44):
    dtdx = 0.3 if solver == "five_point" else 0.5
    return small_case(solver, pusher, n=(nx, 16, 14), dt_over_dx=dtdx, species=(-1.0, 1.0, 0.0))


def _maker(kind, case):
    def make(r, nx):
        return O.Region(nx, case.ny, case.nz, case.dx, case.dx, case.dx, case.dt,
                        solver=SOLVER_ID[case.solver], pusher=PUSHER_ID[case.pusher], seed=7, kind=kind)
    return make


def _box(make, case, fields, parts, n, comm=None, species=None):
    b = S.SlabBox(S.SlabLayout.even(case.nx, n), make, comm)
    b.set_fields([fields[k] for k in FIELD_PLANES])
    b.init_boundaries()
    if species is None:
        b.add_particles(None, all_particles(parts))
    else:
        for s, p in zip(species, parts):
            b.add_particles(s, p)
    return b


# the schedule every slab test runs: plain steps, moving-window steps and a
# load-balancing resize in the middle
SCHEDULE = [(False, False), (True, False), (False, False), (True, True), (False, False), (False, False)]


def _run(b, steps=SCHEDULE):
    rows = []
    for mw, bal in steps:
        rows.append(b.step(1, external_bz=0.3, moving_window=mw)[0])
        if bal:
            b.balance(0.0, 1.0)
    return np.array(rows)


# ----------------------------------------------------------------------------
# layout and load balancing
# ----------------------------------------------------------------------------
def test_even_layout():
    L = S.SlabLayout.even(100, 3)
    # nx = nx_global + nx_ich (n - 1) split evenly, first regions one larger
    assert L.nx == [39, 39, 38] and L.x0 == [0, 31, 62]
    assert [L.diag_range(r) for r in range(3)] == [(0, 35), (4, 35), (4, 38)]
    owned = [L.owned(r) for r in range(3)]
    assert owned == [(0, 35), (35, 66), (66, 100)]
    with pytest.raises(ValueError):
        S.SlabLayout.even(16, 3)
    L2 = S.SlabLayout.from_partition(100, [0, 30, 64])
    assert L2.nx == [38, 42, 36] and L2.x0 == [0, 30, 64]


@needs_ref
def test_balancing_equals_reference():
    rng = np.random.default_rng(5)
    for trial in range(60):
        size = int(rng.integers(40, 400))
        regions = int(rng.integers(2, min(6, size // 16) + 1))
        kind = trial % 3
        if kind == 0:
            w = 256.0 + rng.integers(0, 5000, size).astype(np.float64)
        elif kind == 1:
            w = 256.0 + 1000.0 * np.exp(-((np.arange(size) - rng.uniform(0, size)) / (0.1 * size)) ** 2)
        else:
            w = rng.uniform(0.5, 2.0, size) * rng.choice([1.0, 20.0], size)
        p = S.optimal_partition(w, regions)
        assert p == O.ref_optimal_partition(w, regions, S.NX_ICH), (trial, p)
        assert S.partition_imbalance(w, p) == O.ref_partition_imbalance(w, p, S.NX_ICH)
        old = S.SlabLayout.even(size, regions).x0
        assert S.partition_imbalance(w, old) == O.ref_partition_imbalance(w, old, S.NX_ICH)
        norm = S.normalize_partition(old, p)
        assert norm == O.ref_normalize_partition(old, p, S.NX_ICH)
        S.SlabLayout.from_partition(size, norm)  # a valid layout


def test_optimal_partition_minimises_the_heaviest_region():
    # brute force over every partition of a small box
    rng = np.random.default_rng(2)
    import itertools
    for _ in range(20):
        w = rng.integers(1, 50, 40).astype(np.float64)
        p = S.optimal_partition(w, 3)
        # every layout with side regions of >= 8 layers and a middle one of >= 16
        best = min(max(S.partition_weights(w, [0, a, b]))
                   for a, b in itertools.combinations(range(1, 33), 2) if b - a >= 8)
        S.SlabLayout.from_partition(40, p)
        assert max(S.partition_weights(w, p)) == best


# ----------------------------------------------------------------------------
# slab runs on the CPU checkers
# ----------------------------------------------------------------------------
def _assert_same_box(a, b, msg=""):
    np.testing.assert_array_equal(a.global_fields(), b.global_fields(), err_msg=msg)
    pa, pb = a.global_particles(None), b.global_particles(None)
    for k in pa:
        np.testing.assert_array_equal(pa[k], pb[k], err_msg=f"{msg} {k}")


@needs_ref
@pytest.mark.parametrize("n", [2, 3])
@pytest.mark.parametrize("solver,pusher", [("fdtd", "boris"), ("five_point", "vay"), ("ndfx", "boris")])
def test_slabs_equal_reference_slabs(n, solver, pusher):
    _ensure_port()
    case, fields, parts = _case(solver, pusher)
    port = _box(_maker("port", case), case, fields, parts, n)
    ref = _box(_maker("ref", case), case, fields, parts, n)
    for i, (mw, bal) in enumerate(SCHEDULE):
        dp = port.step(1, external_bz=0.3, moving_window=mw)
        dr = ref.step(1, external_bz=0.3, moving_window=mw)
        np.testing.assert_array_equal(dp, dr)
        if bal:
            assert port.balance(0.0, 1.0) == ref.balance(0.0, 1.0)
            assert port.layout.x0 == ref.layout.x0
        _assert_same_box(port, ref, f"step {i}")


def test_slabs_match_one_region():
    _ensure_port()
    case, fields, parts = _case()
    one = _box(_maker("port", case), case, fields, parts, 1)
    three = _box(_maker("port", case), case, fields, parts, 3)
    d1, d3 = _run(one), _run(three)
    assert three.layout.x0 != S.SlabLayout.even(case.nx, 3).x0  # the resize happened
    # counts exactly, energies to rounding (regions sum in another order)
    np.testing.assert_array_equal(d1[:, 3:6], d3[:, 3:6])
    np.testing.assert_allclose(d3, d1, rtol=1e-11, atol=0)
    f1, f3 = one.global_fields(), three.global_fields()
    assert np.abs(f1 - f3).max() <= 1e-12 * np.abs(f1).max()
    p1, p3 = one.global_particles(None), three.global_particles(None)
    assert p1["x"].size == p3["x"].size
    np.testing.assert_array_equal(p1["cmr"], p3["cmr"])
    for k in ("x", "y", "z", "ux", "uy", "uz", "g"):
        assert np.abs(p1[k] - p3[k]).max() <= 1e-11 * max(1.0, np.abs(p1[k]).max()), k


def test_layer_counts_and_weights():
    _ensure_port()
    case, fields, parts = _case()
    one = _box(_maker("port", case), case, fields, parts, 1)
    three = _box(_maker("port", case), case, fields, parts, 3)
    counts = np.bincount(all_particles(parts)["x"].astype(int), minlength=case.nx)
    np.testing.assert_array_equal(one.regions[0].layer_counts(), counts)
    w = case.ny * case.nz + 2.0 * counts
    np.testing.assert_array_equal(one.layer_weights(2.0), w)
    np.testing.assert_array_equal(three.layer_weights(2.0), w)


# ----------------------------------------------------------------------------
# torch.distributed (gloo) ranks, one region each
# ----------------------------------------------------------------------------
def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gloo_worker(rank, world, port, out_dir):
    import datetime
    import sys
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from oracle import oracle as O_
        from quill_b200 import slabs as S_
        from tests import test_slabs as T
        case, fields, parts = T._case()
        b = T._box(T._maker("port", case), case, fields, parts, world, comm=S_.TorchComm("cpu"))
        rows = T._run(b)
        reg = b.regions[rank]
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), rows=rows, fields=reg.get_fields(),
                 x0=np.array(b.layout.x0), **{f"p_{k}": v for k, v in reg.get_particles().items()})
        assert isinstance(reg, O_.Region)
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_equal_in_process(world):
    _ensure_port()
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    port = _free_port()
    with tempfile.TemporaryDirectory() as d:
        procs = [ctx.Process(target=_gloo_worker, args=(r, world, port, d)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=240)
            assert p.exitcode == 0
        case, fields, parts = _case()
        local = _box(_maker("port", case), case, fields, parts, world)
        rows = _run(local)
        for r in range(world):
            z = np.load(os.path.join(d, f"rank{r}.npz"))
            np.testing.assert_array_equal(z["rows"], rows)
            np.testing.assert_array_equal(z["x0"], local.layout.x0)
            np.testing.assert_array_equal(z["fields"], local.regions[r].get_fields())
            lp = local.regions[r].get_particles()
            for k in lp:
                np.testing.assert_array_equal(z[f"p_{k}"], lp[k])


# ----------------------------------------------------------------------------
# library regions on the GPU
# ----------------------------------------------------------------------------
def _gpu_maker(case, precision="fp64"):
    from quill_b200.api import Region

    def make(r, nx):
        return Region(nx, case.ny, case.nz, case.dx, case.dx, case.dx, case.dt, species_cmr=(-1.0, 1.0, 0.0),
                      solver=case.solver, pusher=case.pusher, precision=precision)
    return make


@pytest.mark.gpu
@pytest.mark.parametrize("device_payloads", [False, True])
@pytest.mark.parametrize("solver,pusher", [("fdtd", "boris"), ("five_point", "vay")])
def test_gpu_slabs_equal_checker_slabs(solver, pusher, device_payloads):
    if not gpu_available():
        pytest.skip("needs a CUDA device")
    _ensure_port()
    case, fields, parts = _case(solver, pusher)
    comm = S.LocalComm("cuda:0" if device_payloads else None)
    gpu = _box(_gpu_maker(case), case, fields, parts, 3, comm=comm, species=(0, 1, 2))
    cpu = _box(_maker("port", case), case, fields, parts, 3)
    for i, (mw, bal) in enumerate(SCHEDULE):
        dg = gpu.step(1, external_bz=0.3, moving_window=mw)[0]
        dc = cpu.step(1, external_bz=0.3, moving_window=mw)[0]
        np.testing.assert_array_equal(dg[3:6], dc[3:6])
        np.testing.assert_allclose(dg, dc, rtol=1e-12, atol=0, err_msg=f"step {i}")
        if bal:
            assert gpu.balance(0.0, 1.0) == cpu.balance(0.0, 1.0)
        fg, fc = gpu.global_fields(), cpu.global_fields()
        assert np.abs(fg - fc).max() <= 1e-12 * np.abs(fc).max(), i
        pc = cpu.global_particles(None)
        for s, cmr in enumerate((-1.0, 1.0, 0.0)):
            pg = gpu.global_particles(s)
            sel = pc["cmr"] == cmr
            assert pg["x"].size == sel.sum(), (i, s)
            for k in ("x", "y", "z", "ux", "uy", "uz", "g", "q"):
                np.testing.assert_allclose(pg[k], pc[k][sel], rtol=1e-12, atol=1e-12, err_msg=f"{i} {s} {k}")
    np.testing.assert_array_equal(gpu.regions[1].layer_counts(), cpu.regions[1].layer_counts())
    gpu.close()


@pytest.mark.gpu
def test_gpu_mixed_slabs_match_one_region():
    if not gpu_available():
        pytest.skip("needs a CUDA device")
    case, fields, parts = _case()
    one = _box(_gpu_maker(case, "mixed"), case, fields, parts, 1, species=(0, 1, 2))
    three = _box(_gpu_maker(case, "mixed"), case, fields, parts, 3, species=(0, 1, 2))
    d1, d3 = _run(one), _run(three)
    # FP32 offsets move between frames without rounding; J atomics differ
    np.testing.assert_allclose(d3, d1, rtol=2e-4, atol=0)
    f1, f3 = one.global_fields(), three.global_fields()
    assert np.abs(f1 - f3).max() <= 1e-4 * np.abs(f1).max()
    one.close()
    three.close()


def _cell_sorted(rng, m, lo, hi, ny, nz):
    """m particles with x in [lo, hi), sorted by cell, random order inside a
    cell kept (stable sort)."""
    p = {"x": rng.uniform(lo, hi, m), "y": rng.uniform(0, ny, m), "z": rng.uniform(0, nz, m),
         "ux": rng.normal(0, 0.1, m), "uy": rng.normal(0, 0.1, m), "uz": rng.normal(0, 0.1, m), "q": rng.uniform(-2, -1, m)}
    p["g"] = np.sqrt(1 + p["ux"] ** 2 + p["uy"] ** 2 + p["uz"] ** 2)
    cell = (p["x"].astype(int) * ny + p["y"].astype(int)) * nz + p["z"].astype(int)
    o = np.argsort(cell, kind="stable")
    return {k: v[o] for k, v in p.items()}


@pytest.mark.gpu
@pytest.mark.parametrize("device_payload", [False, True])
@pytest.mark.parametrize("end", ["low", "high"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_gpu_end_slab_replacement_follows_the_list_rule(precision, end, device_payload):
    """Replacing the particles of a slab at either x end (the halo update of
    the exchange) empties the slab's cells and puts the given particles in
    them in the given order: the traversal becomes new + kept (low end) or
    kept + new (high end).  The same holds when an input particle lies
    outside the slab (it then joins the head of its cell, as a load does)."""
    if not gpu_available():
        pytest.skip("needs a CUDA device")
    import torch
    from quill_b200.api import Region
    nx, ny, nz, w = 20, 6, 5, 3
    rng = np.random.default_rng(11)
    reg = Region(nx, ny, nz, 0.1, 0.1, 0.1, 0.05, species_cmr=(-1.0,), solver="fdtd", pusher="boris",
                 precision=precision)
    reg.add_particles(0, _cell_sorted(rng, 4000, 0, nx, ny, nz))
    before = reg.get_particles(0)
    i0 = 0 if end == "low" else nx - w
    new = _cell_sorted(rng, 700, i0, i0 + w, ny, nz)
    payload = {k: torch.from_numpy(v).cuda() for k, v in new.items()} if device_payload else new
    reg.replace_particle_slab(0, i0, w, payload)
    after = reg.get_particles(0)
    inside = (before["x"] >= i0) & (before["x"] < i0 + w)
    kept = {k: before[k][~inside] for k in ("x", "y", "z", "ux", "uy", "uz", "g", "q")}
    want = {k: (np.concatenate([new[k], kept[k]]) if end == "low" else np.concatenate([kept[k], new[k]]))
            for k in kept}
    assert after["x"].size == want["x"].size
    tol = 0 if precision == "fp64" else 2e-6
    for k in want:
        np.testing.assert_allclose(after[k], want[k], rtol=tol, atol=tol * nx, err_msg=k)
    # a particle outside the slab: loaded into its own cell, at its head
    stray = _cell_sorted(rng, 5, i0, i0 + w, ny, nz)
    stray["x"][-1] = 10.5
    before = reg.get_particles(0)
    reg.replace_particle_slab(0, i0, w, stray)
    after = reg.get_particles(0)
    assert after["x"].size == before["x"].size - 700 + 5
    assert np.isclose(after["x"], 10.5, rtol=0, atol=tol * nx + 1e-12).sum() == 1
    reg.step(1)  # the new layout steps (layers 0, n-2, n-1 are erased first)
    assert 0 < reg.count(0) <= after["x"].size
    reg.close()
