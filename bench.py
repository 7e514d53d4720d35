"""Throughput of QUILL's per-timestep PIC loop on B200 (one JSON line).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config cfg5_512_fdtd_boris] [--grid NX NY NZ]

Workload: the 512^3-cell, 4-ppc configuration (dx = lambda/20, dt = dx/2,
FDTD solver, Boris pusher, QED off, uniform 0.05 n_cr electron plasma with
10 keV Maxwellian momenta, linearly polarised a0 = 20 laser pulse): 5.25e8
electrons, 1.34e8 cells.  Synthetic, seeded, generated on the GPU.

A step is one full timestep of main.cpp:2321-2331 (push + deposition +
rebin, diagnostics, Maxwell solver + Bbar).  `value` = particle-steps/s with
the state resident in HBM; FP64 (the reference arithmetic) is the headline,
the mixed-precision run is reported in `mixed`.  `e2e` = the same metric for
the whole job through the C ABI from pinned host buffers (create, load
fields and particles, K steps with the per-step diagnostics copied to the
host, dump of the fields to the host).  Inputs (tens of GB) are far larger
than L2, so no flush is needed between steps.

`--impl reference` times the reference's own CPU build (oracle/_ref) on the
host cores, stepping the same box: cut into x-slab regions as the reference
cuts it for its MPI ranks, one host process per region and core (the
exchange between the regions is left out: no MPI on the host).
"""
from __future__ import annotations

import argparse
import json
import math
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAK_FALLBACK_GBS = 6650.0


METRIC = "particle-steps/s & field cell-updates/s, FP64 vs mixed, 1 B200, at stated drift"


def workload_config(case):
    """The `config` of both arms' lines: the workload, nothing that differs
    between them."""
    sp = case.species[0]
    # particles per cell: one figure for one species, per species for several
    ppc = " + ".join(str(x.ppc) for x in case.species)
    return {"workload": f"{case.name}: {case.nx}x{case.ny}x{case.nz} cells, dx=lambda/{round(1 / case.dx_lambda)}, "
                        f"dt={case.dt_over_dx:g}dx, {case.solver.upper()} + {case.pusher}, "
                        f"QED {'on' if case.qed else 'off'}, {ppc} ppc at {sp.n0:g} n_cr, "
                        f"T={sp.theta / 1.957e-3:g} keV, laser a0={case.laser.a0:g}",
            "l2_flush": "not needed: particle and field arrays exceed L2"}


def hbm_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return PEAK_FALLBACK_GBS, "fallback"


# algorithmic bytes per particle-step and per cell-update (push kernel reads
# x y z ux uy uz g q and writes all but q; the fused field step reads E B J,
# writes E B Bbar, the deposit flush writes J once)
BYTES = {"fp64": (120, 168), "mixed": (68, 84)}
# DRAM traffic of one push launch per particle (dram__bytes_read.sum +
# dram__bytes_write.sum over the particles of the launch), from an ncu
# capture of one k_push64 / k_push32 launch on the same physics at 160^3
# (15,250,622 particles, about 2.5 GB on the device).  At fixed ppc the
# traffic grows in proportion to the particle count, so the per-particle
# figure is scaled by Np for the grid being measured.
TRAFFIC_PER_PARTICLE = {"fp64": (1.361e9 + 1.120e9) / 15250622,
                        "mixed": (0.783e9 + 0.645e9) / 15250622}
TRAFFIC_SOURCE = "ncu capture of one launch at 160^3 (same physics), per particle x Np"


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=10)
        except Exception:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------------------
# CPU side: the reference build on the same workload
# ----------------------------------------------------------------------------
# The reference's only parallelism is its cut of the box into x-slab regions,
# one per MPI rank (main.cpp:2232-2267), neighbours overlapping by 8 cells.
# Here each host process is one such region of the benchmark box, built by
# the reference's own code (oracle/_ref, Release flags): its slab of the
# laser fields and its slab of the plasma, its diagnostics over the cells it
# owns.  The regions step concurrently; what is left out is the MPI exchange
# of halos and crossing particles between steps (no MPI on the host).

def _ref_region_job(job, barrier, queue):
    """One x-slab region of the workload on one host core: build, warm up,
    wait for the other regions, time `steps` steps.  Puts (region, units,
    cell-updates, t0, t1, particles, error) on the queue."""
    kind, cfg_name, grid, nreg, r, steps, warm, seed = job
    try:
        sys.path.insert(0, ROOT)
        import numpy as np
        from oracle import oracle as O
        from quill_b200 import workloads as W
        from quill_b200.slabs import SlabLayout
        case = W.config(cfg_name)
        if grid:
            case = W.scaled(case, *grid)
        lay = SlabLayout.even(case.nx, nreg)
        x0, nxr = lay.x0[r], lay.nx[r]
        solver = {"fdtd": 0, "ndfx": 1, "five_point": 2}[case.solver]
        pusher = {"vay": 0, "boris": 1}[case.pusher]
        icmr = tuple(sp.cmr for sp in case.species if sp.cmr not in (-1.0, 1.0, 0.0))
        reg = O.Region(nxr, case.ny, case.nz, case.dx, case.dx, case.dx, case.dt, solver=solver, pusher=pusher,
                       icmr=icmr, kind=kind, flavour="fast")
        f = W.make_fields(case, x0, nxr)
        reg.set_fields(*[f[k] for k in ("ex", "ey", "ez", "bx", "by", "bz")])
        del f
        reg.init_boundaries()
        rng = np.random.default_rng(seed + r)
        for sp in case.species:
            for part in W.particle_layers(case, sp, rng, x0, nxr):
                reg.add_particles(part)
        lo, hi = lay.diag_range(r)
        reg.set_diag_range(lo, hi)
        if warm:
            reg.step(warm)
        d0 = reg.compute_diag()
        barrier.wait(timeout=1800)
        t0 = time.monotonic()
        d = reg.step(steps)
        t1 = time.monotonic()

        def count(row):  # N_qp_e + N_qp_p + N_qp_g + ions (the diagnostic row layout)
            return float(row[3] + row[4] + row[5] + sum(row[10 + 2 * m] for m in range(reg.n_ion)))

        units = count(d0) + sum(count(row) for row in d[:-1])
        queue.put((r, units, (hi - lo) * case.ny * case.nz * steps, t0, t1, reg.count(), None))
    except Exception as e:  # reported by the parent
        try:
            barrier.abort()
        except Exception:
            pass
        queue.put((r, 0.0, 0, 0.0, 0.0, 0, f"{type(e).__name__}: {e}"))


def cpu_kind():
    from oracle import oracle as O
    return "reference" if O.available("ref", "fast") else "port"


def _mem_available_bytes():
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    return int(line.split()[1]) * 1024
    except OSError:
        pass
    return None


def run_reference_regions(cfg_name, grid, nreg, steps, warm, regions=None):
    """The reference stepping regions `regions` (default: all) of the
    workload cut into `nreg` x-slabs, one process each, concurrently.
    Returns the units over the common timed window."""
    import multiprocessing as mp
    kind = "ref" if cpu_kind() == "reference" else "port"
    regions = list(range(nreg)) if regions is None else list(regions)
    ctx = mp.get_context("spawn")
    barrier = ctx.Barrier(len(regions))
    q = ctx.Queue()
    procs = [ctx.Process(target=_ref_region_job, args=((kind, cfg_name, grid, nreg, r, steps, warm, 1000), barrier, q))
             for r in regions]
    for pr in procs:
        pr.start()
    res = []
    for _ in procs:
        res.append(q.get(timeout=3600))
    for pr in procs:
        pr.join()
    errs = [x[6] for x in res if x[6]]
    if errs:
        raise RuntimeError("reference region failed: " + errs[0])
    t = max(x[4] for x in res) - min(x[3] for x in res)
    units = sum(x[1] for x in res)
    cells = sum(x[2] for x in res)
    return {"particle_steps_per_s": units / t, "cell_updates_per_s": cells / t, "seconds": t,
            "particles": sum(x[5] for x in res), "kind": cpu_kind(), "procs": len(regions), "regions": nreg,
            "steps": steps, "units": units}


def reference_bytes_estimate(case, nreg):
    """Host memory of the reference's regions: about 104 B per particle
    (its particle record, containers.h:54-66) and 112 B per cell (list
    heads and the four field3d arrays), overlaps included, plus the
    generator's transient arrays."""
    ppc = sum(sp.ppc for sp in case.species)
    cells = (case.nx + 8 * (nreg - 1)) * case.ny * case.nz
    return cells * (112 + 104 * ppc) + nreg * (1 << 30)


# ----------------------------------------------------------------------------
# GPU side
# ----------------------------------------------------------------------------

def build_region(case, precision, device_index, planes_per_chunk=48):
    import torch
    from quill_b200 import workloads as W
    from quill_b200.api import Region
    f = W.make_fields_torch(case, device=f"cuda:{device_index}")
    reg = Region(case.nx, case.ny, case.nz, case.dx, case.dx, case.dx, case.dt,
                 species_cmr=tuple(sp.cmr for sp in case.species), solver=case.solver, pusher=case.pusher,
                 precision=precision, device=device_index)
    reg.set_stream(torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    reg.lib.qp_load_fields(reg.h, *[_tp(f[k]) for k in ("ex", "ey", "ez", "bx", "by", "bz")])
    del f
    reg.init_boundaries()
    for si, sp in enumerate(case.species):
        for ch in W.particle_chunks_torch(case, sp, planes_per_chunk, device=f"cuda:{device_index}",
                                          seed=case.seed + 17 * si):
            _load_torch(reg, si, ch)
            del ch
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    return reg


def _tp(t):
    import ctypes as C
    return C.cast(t.data_ptr(), C.POINTER(C.c_double))


def _load_torch(reg, si, ch):
    keys = ("x", "y", "z", "ux", "uy", "uz", "g", "q")
    r = reg.lib.qp_load_particles(reg.h, si, ch["x"].numel(), *[_tp(ch[k]) for k in keys], None)
    reg._check(r)


def reduce_over_ranks(dist, ms, units, device):
    """Replicas: the job's time is the slowest rank's, its units the sum over
    ranks (every rank takes the same two collectives)."""
    if dist is None:
        return ms, units
    import torch
    x = torch.tensor([ms], device=device, dtype=torch.float64)
    dist.all_reduce(x, op=dist.ReduceOp.MAX)
    y = torch.tensor([float(units)], device=device, dtype=torch.float64)
    dist.all_reduce(y)
    return float(x.item()), float(y.item())


def total_energy(d):
    return d.energy_f + d.energy_e + d.energy_p + d.energy_ph + sum(d.ienergy[m] for m in range(d.n_ion))


def time_region(reg, steps, warmup, device_index):
    """Device-resident timing of `steps` steps after `warmup` steps."""
    import torch
    diags = reg.step(warmup) if warmup else []
    reg.set_timing(True)
    l0 = reg.launch_count()
    n_before = sum(reg.count(i) for i in range(reg.n_species))
    clk = Clocks(device_index)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clk.start()
    time.sleep(0.3)
    e0.record()
    d = reg.step(steps)
    e1.record()
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms = e0.elapsed_time(e1)
    launches = reg.launch_count() - l0
    phase_ms, nst = reg.get_timing()
    reg.set_timing(False)
    n_after = sum(reg.count(i) for i in range(reg.n_species))
    psteps = sum(sum(x.n_macro[i] for i in range(reg.n_species)) for x in d)
    # particles pushed per step are those alive at its start: n_before, then
    # the counts after each step
    pushed = n_before + sum(sum(x.n_macro[i] for i in range(reg.n_species)) for x in d[:-1])
    return {"ms": ms, "steps": steps, "pushed": pushed, "launches": launches, "phase_ms": list(phase_ms),
            "clocks": clocks, "diags": diags + d, "n_after": n_after}


def e2e_run(case, precision, steps, device_index, host):
    """Whole job through the C ABI from pinned host buffers."""
    import ctypes as C
    import numpy as np
    import torch
    from quill_b200.api import Diag, Region
    t0 = time.perf_counter()
    # the particle counts are known up front: size the stores once
    reg = Region(case.nx, case.ny, case.nz, case.dx, case.dx, case.dx, case.dt,
                 species_cmr=tuple(sp.cmr for sp in case.species), solver=case.solver, pusher=case.pusher,
                 precision=precision, device=device_index,
                 capacity=[p["x"].numel() for p in host["p"]])
    lib = reg.lib
    t1 = time.perf_counter()
    reg._check(lib.qp_load_fields(reg.h, *[C.cast(host["f"][k].data_ptr(), C.POINTER(C.c_double))
                                           for k in ("ex", "ey", "ez", "bx", "by", "bz")]))
    reg.init_boundaries()
    t2 = time.perf_counter()
    keys = ("x", "y", "z", "ux", "uy", "uz", "g", "q")
    h2d = sum(host["f"][k].numel() * 8 for k in host["f"])
    for si, p in enumerate(host["p"]):
        reg._check(lib.qp_load_particles(reg.h, si, p["x"].numel(),
                                         *[C.cast(p[k].data_ptr(), C.POINTER(C.c_double)) for k in keys], None))
        h2d += sum(p[k].numel() * 8 for k in keys)
    diag = (Diag * steps)()
    pushed = sum(reg.count(i) for i in range(reg.n_species))
    t3 = time.perf_counter()
    reg._check(lib.qp_step(reg.h, steps, 0.0, diag))
    t4 = time.perf_counter()
    pushed += sum(sum(diag[s].n_macro[i] for i in range(reg.n_species)) for s in range(steps - 1))
    # the job's field output: the slices the reference's writers produce
    out = host["out"]
    reg._check(lib.qp_dump_field_slices(reg.h, case.nx // 2, C.cast(out.data_ptr(), C.POINTER(C.c_double))))
    reg.close()
    t = time.perf_counter() - t0
    d2h = steps * C.sizeof(Diag) + out.numel() * 8
    return {"value": pushed / t, "seconds": t, "steps": steps, "h2d_bytes_per_step": h2d // steps,
            "d2h_bytes_per_step": d2h // steps,
            "phases_s": {"create": t1 - t0, "load_fields": t2 - t1, "load_particles": t3 - t2, "steps": t4 - t3,
                         "dump_and_destroy": t0 + t - t4}}


def pinned_host_state(case, device_index):
    """Generate the state on the GPU and copy it to pinned host memory (not
    timed)."""
    import torch
    from quill_b200 import workloads as W
    f = W.make_fields_torch(case, device=f"cuda:{device_index}")
    hf = {k: v.cpu().pin_memory() for k, v in f.items()}
    del f
    hp = []
    for si, sp in enumerate(case.species):
        # one pinned array per component: sizes from a first pass of the
        # generator, then the chunks copied into place
        dev, seed = f"cuda:{device_index}", case.seed + 17 * si
        m = sum(ch["x"].numel() for ch in W.particle_chunks_torch(case, sp, 48, device=dev, seed=seed))
        arrs = None
        o = 0
        for ch in W.particle_chunks_torch(case, sp, 48, device=dev, seed=seed):
            if arrs is None:
                arrs = {k: torch.empty(m, dtype=torch.float64).pin_memory() for k in ch}
            k_n = ch["x"].numel()
            for k, v in ch.items():
                arrs[k][o:o + k_n].copy_(v)
            o += k_n
        hp.append(arrs)
    out = torch.empty(12 * (case.nx * (case.ny + case.nz) + case.ny * case.nz), dtype=torch.float64).pin_memory()
    torch.cuda.empty_cache()
    return {"f": hf, "p": hp, "out": out}


def slab_main(args, case, rank, world, local):
    """One box of world x local_regions x-slab regions, each the size of the
    benchmark box along x (weak scaling), stepped with the neighbour exchange
    of synchronize_regions (main.cpp:1493-1506) after every step."""
    import datetime
    import torch
    from quill_b200 import workloads as W
    from quill_b200.api import Region
    from quill_b200.slabs import NM, LocalComm, SlabBox, SlabLayout, TorchComm
    dist = None
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    stream = torch.cuda.Stream(device=local)
    torch.cuda.set_stream(stream)
    dev = f"cuda:{local}"
    nreg = world * args.local_regions
    gcase = W.scaled(case, case.nx * nreg, case.ny, case.nz)
    gcase.seed = 1234
    layout = SlabLayout.even(gcase.nx, nreg)
    if world > 1:
        if args.local_regions != 1:
            raise SystemExit("--local-regions needs a single process")
        comm = TorchComm(device=dev)
    else:
        comm = LocalComm(device=dev)
    prec = "fp64"
    species = tuple(sp.cmr for sp in gcase.species)

    def make_region(r, nxl):
        reg = Region(nxl, gcase.ny, gcase.nz, gcase.dx, gcase.dx, gcase.dx, gcase.dt, species_cmr=species,
                     solver=gcase.solver, pusher=gcase.pusher, precision=prec, device=local)
        reg.set_stream(stream.cuda_stream)
        return reg

    box = SlabBox(layout, make_region, comm)
    keys = ("x", "y", "z", "ux", "uy", "uz", "g", "q")
    for r in box.local:
        reg, x0, nxl = box.regions[r], layout.x0[r], layout.nx[r]
        f = W.make_fields_torch(gcase, device=dev, i0=x0, nxr=nxl)
        torch.cuda.synchronize()
        reg._check(reg.lib.qp_load_fields(reg.h, *[_tp(f[k]) for k in ("ex", "ey", "ez", "bx", "by", "bz")]))
        del f
        for si, sp in enumerate(gcase.species):
            for ch in W.particle_chunks_torch(gcase, sp, 48, device=dev, seed=gcase.seed + 17 * si + 1000 * r,
                                              i_range=(x0, x0 + nxl)):
                _load_torch(reg, si, ch)
                del ch
    box.init_boundaries()
    torch.cuda.synchronize()
    torch.cuda.empty_cache()

    def count(row):  # N_qp_e + N_qp_p + N_qp_g + ions
        return float(row[3] + row[4] + row[5] + sum(row[10 + 2 * m] for m in range((len(row) - 10) // 2)))

    rows = box.step(args.warmup) if args.warmup else []
    last = count(rows[-1]) if len(rows) else None
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * args.steps + 1)]
    ev[0].record(stream)
    pushed = 0.0
    for k in range(args.steps):
        acc = None
        for r in box.local:
            d = box.regions[r].step(1)[0].as_array()
            acc = d if acc is None else acc + d
        ev[2 * k + 1].record(stream)
        row = comm.allsum(acc)
        box.synchronize(NM, NM)
        ev[2 * k + 2].record(stream)
        pushed += last if last is not None else count(row)
        last = count(row)
    torch.cuda.synchronize()
    ms = ev[0].elapsed_time(ev[-1])
    exch = sum(ev[2 * k + 1].elapsed_time(ev[2 * k + 2]) for k in range(args.steps))
    if dist:
        t = torch.tensor([ms, exch], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, exch = float(t[0]), float(t[1])
        dist.barrier()
        for reg in box.regions.values():
            reg.close()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": pushed / (ms * 1e-3), "unit": "particle-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded, generated on the GPU)",
        "cell_updates_per_s": gcase.nx * gcase.ny * gcase.nz * args.steps / (ms * 1e-3),
        "config": workload_config(case),
        "parallelism": f"one box of {nreg} x-slab regions of {case.nx} cells along x ({gcase.nx}x{gcase.ny}x"
                       f"{gcase.nz} cells), {world} GPU(s); neighbours exchange field halos and particles after "
                       f"every step ({'NCCL point to point' if world > 1 else 'device copies in one process'})",
        "exchange_ms_per_step": exch / args.steps,
        "regions_per_gpu": args.local_regions,
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="cfg5_512_fdtd_boris")
    ap.add_argument("--grid", type=int, nargs=3, default=None)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--cpu-steps", type=int, default=2)
    ap.add_argument("--ref-regions", type=int, default=0,
                    help="x-slab regions of the reference runs (default: the host's core count)")
    ap.add_argument("--mode", default="replicas", choices=["replicas", "slabs"],
                    help="replicas: one independent box per GPU; slabs: one box cut into x-slab regions, one "
                         "region per GPU (the reference's decomposition), neighbours exchanging halos and "
                         "particles every step over NCCL")
    ap.add_argument("--local-regions", type=int, default=1,
                    help="slabs mode: regions per process (several on one GPU measure the exchange without NVLink)")
    ap.add_argument("--drift-steps", type=int, default=1000,
                    help="also run this many untimed steps per precision and report the relative drift of the "
                         "total energy (field + particles) over them")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    from quill_b200 import workloads as W
    case = W.config(args.config)
    if args.grid:
        case = W.scaled(case, *args.grid)
    nc = case.nx * case.ny * case.nz

    if args.impl == "reference":
        if rank != 0:
            return
        nreg = args.ref_regions or (os.cpu_count() or 1)
        need, have = reference_bytes_estimate(case, nreg), _mem_available_bytes()
        regions = None
        if have is not None and need > 0.8 * have:
            # not enough host memory for every region: a bounded sample of
            # the regions, their units only
            per = need / nreg
            regions = list(range(max(1, int(0.8 * have // per))))
        r = run_reference_regions(args.config, args.grid, nreg, args.steps, args.warmup, regions)
        sample = (f"all {nreg} x-slab regions of the box (the reference's own decomposition, n_sr = {nreg}, "
                  f"neighbours overlapping by 8 cells), one process each, stepped concurrently; "
                  f"{r['particles']} particles held (overlaps included); no halo exchange between steps")
        if regions is not None:
            sample = (f"regions 0..{len(regions) - 1} of the box's {nreg} x-slab regions (host memory for "
                      f"{len(regions)}), one process each; their particle-steps only")
        line = {
            "impl": "reference", "metric": METRIC, "value": r["particle_steps_per_s"], "unit": "particle-steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * r["seconds"] / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "cell_updates_per_s": r["cell_updates_per_s"],
            "config": workload_config(case),
            "parallelism": f"{r['procs']} host processes (one x-slab region each)",
            "cpu_baseline": {"value": r["particle_steps_per_s"], "unit": "particle-steps/s", "cores": r["procs"],
                             "kind": r["kind"], "sample": sample},
            "e2e": {"value": r["particle_steps_per_s"], "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line), flush=True)
        return

    if args.mode == "slabs":
        slab_main(args, case, rank, world, local)
        return

    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local)
    dev = local
    # one stream for torch (generation) and the library (qp_set_stream), so
    # that the library's copies are ordered after the generating kernels
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    case.seed = 1234 + rank

    peak, peak_kind = hbm_peak()
    results = {}
    for prec in (["fp64"] if args.no_mixed else ["fp64", "mixed"]):
        reg = build_region(case, prec, dev)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        t = time_region(reg, args.steps, args.warmup, dev)
        f_end = torch.empty((12, case.nx, case.ny, case.nz), dtype=torch.float64, device=f"cuda:{dev}")
        reg._check(reg.lib.qp_dump_fields(reg.h, _tp(f_end)))
        t["fields_end"] = f_end[:6].clone()
        del f_end
        reg.close()
        del reg
        torch.cuda.empty_cache()
        ms, pushed_all = reduce_over_ranks(dist, t["ms"], t["pushed"], f"cuda:{dev}")
        bp, bc = BYTES[prec]
        np_avg = t["pushed"] / t["steps"]
        push_ms = t["phase_ms"][0] / t["steps"]
        achieved = np_avg * bp / (push_ms * 1e-3) / 1e9
        d = t["diags"]
        w0, w1 = total_energy(d[0]), total_energy(d[-1])
        results[prec] = {
            "value": pushed_all / (ms * 1e-3),
            "cell_updates_per_s": world * nc * t["steps"] / (ms * 1e-3),
            "ms_per_step": ms / t["steps"],
            "gpu_launches": t["launches"],
            "phase_ms_per_step": {k: v / t["steps"] for k, v in zip(("push_deposit", "rebin", "fields", "diag"),
                                                                     t["phase_ms"])},
            "roofline": {"kernel": "push_deposit (k_push64)" if prec == "fp64" else "push_deposit (k_push32)",
                         "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": np_avg * TRAFFIC_PER_PARTICLE[prec],
                         "traffic_source": TRAFFIC_SOURCE,
                         "algorithmic_bytes_per_launch": np_avg * bp},
            "step_roofline_frac": (np_avg * bp + nc * bc) / (ms * 1e-3 / t["steps"]) / 1e9 / peak,
            "energy_drift": (w1 - w0) / w0 if w0 else None,
            "drift_steps": len(d),
            "clocks": t["clocks"],
            "fields_end": t["fields_end"],
            "particles": t["n_after"],
        }
    # long untimed runs for the energy drift (opt-in)
    if args.drift_steps > 0:
        drift_fields = {}
        for prec in results:
            reg = build_region(case, prec, dev)
            reg.set_erased_tracking(True)
            w, closed, lost = [], [], 0.0
            left = args.drift_steps
            while left > 0:
                k = min(left, 50)
                for x in reg.step(k):
                    lost += x.energy_erased
                    w.append(total_energy(x))
                    closed.append(w[-1] + lost)
                left -= k
            f_end = torch.empty((12, case.nx, case.ny, case.nz), dtype=torch.float64, device=f"cuda:{dev}")
            reg._check(reg.lib.qp_dump_fields(reg.h, _tp(f_end)))
            drift_fields[prec] = f_end[:6].clone()
            del f_end
            reg.close()
            del reg
            torch.cuda.empty_cache()
            results[prec]["long_run_energy_drift"] = {
                "steps": args.drift_steps,
                "relative_drift": (w[-1] - w[0]) / w[0],
                "max_relative_excursion": max(abs(x - w[0]) for x in w) / w[0],
                "relative_drift_with_erased": (closed[-1] - closed[0]) / closed[0],
                "max_relative_excursion_with_erased": max(abs(x - closed[0]) for x in closed) / closed[0],
                "note": "relative_drift is the total energy of the energy output (field + particles), which "
                        "particles leaving through the absorbing p_boundary layers lower; the _with_erased "
                        "figures add the energy those particles carried off (closed balance)"}
    if args.drift_steps > 0 and "mixed" in results:
        a, b = results["mixed"]["long_run_energy_drift"], results["fp64"]["long_run_energy_drift"]
        a["drift_minus_fp64"] = a["relative_drift_with_erased"] - b["relative_drift_with_erased"]
        x, y = drift_fields["mixed"], drift_fields["fp64"]
        a["field_rel_l2_vs_fp64"] = float(torch.linalg.vector_norm(x - y) / torch.linalg.vector_norm(y))
    if args.drift_steps > 0:
        del drift_fields
        torch.cuda.empty_cache()
    # mixed vs FP64 field error after the same steps from the same state
    if "mixed" in results:
        a, b = results["mixed"]["fields_end"], results["fp64"]["fields_end"]
        results["mixed"]["field_rel_l2_vs_fp64"] = float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))
    for r in results.values():
        r.pop("fields_end", None)

    e2e = None
    if not args.no_e2e:
        host = pinned_host_state(case, dev)
        # one untimed 1-step job first, as the device timing has warm-up
        # steps: the first job of a process pays one-time driver costs (its
        # particle upload ran at about 20 GB/s, every later one at the link's
        # 54 GB/s)
        e2e_run(case, "fp64", 1, dev, host)
        e2e = e2e_run(case, "fp64", args.steps, dev, host)
        del host
        if dist:
            sec, units = reduce_over_ranks(dist, e2e["seconds"], e2e["value"] * e2e["seconds"], f"cuda:{dev}")
            e2e["value"] = units / sec

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        # one core: one x-slab region of the box (the one the laser enters)
        # for a bounded sample of steps
        nreg = args.ref_regions or (os.cpu_count() or 1)
        c = run_reference_regions(args.config, args.grid, nreg, args.cpu_steps, 1, regions=[0])
        cpu = {"value": c["particle_steps_per_s"], "unit": "particle-steps/s", "cores": 1, "kind": c["kind"],
               "sample": f"region 0 of the box cut into {nreg} x-slab regions (the reference's decomposition; "
                         f"{c['particles']} particles), {c['steps']} steps after 1 warm-up step, "
                         f"{c['seconds']:.1f} s",
               "cell_updates_per_s": c["cell_updates_per_s"], "host_cores_total": os.cpu_count()}

    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    f64 = results["fp64"]
    line = {
        "metric": METRIC, "value": f64["value"], "unit": "particle-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": f64["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded, generated on the GPU)",
        "cell_updates_per_s": f64["cell_updates_per_s"],
        "config": workload_config(case),
        "particles": f64["particles"],
        "parallelism": "1 GPU" if world == 1 else f"{world} independent replicas (one region per GPU)",
        "roofline": f64["roofline"], "step_roofline_frac": f64["step_roofline_frac"],
        "energy_drift": f64["energy_drift"], "drift_steps": f64["drift_steps"],
        "phase_ms_per_step": f64["phase_ms_per_step"],
        "clocks": f64["clocks"], "gpu_launches": f64["gpu_launches"],
        "long_run_energy_drift": f64.get("long_run_energy_drift"),
        "mixed": {k: v for k, v in results.get("mixed", {}).items() if k != "clocks"} or None,
        "e2e": ({"value": e2e["value"], "unit": "particle-steps/s", "h2d_bytes_per_step": e2e["h2d_bytes_per_step"],
                 "d2h_bytes_per_step": e2e["d2h_bytes_per_step"], "seconds": e2e["seconds"],
                 "phases_s": e2e["phases_s"],
                 "includes": "qp_create, field + particle load from pinned host memory, K steps with per-step "
                             "diagnostics to host, the field output slices to host, qp_destroy; after one untimed "
                             "1-step job"}
                if e2e else None),
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
