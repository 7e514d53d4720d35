"""The QED cascade of the benchmark's third configuration on one GPU.

    python -m quill_b200.cascade [--grid 256 256 256] [--steps 600]
                                 [--precision fp64|mixed] [--seed 0] [--every 50]
                                 [--crpc 1.5]

Five-point solver, Vay pusher, QED on (photon emission, Breit-Wheeler pairs,
vacuum pairs): two counter-propagating circularly polarised pulses (a0 =
1500, 10 lambda FWHM, 3 lambda waist; the second is the first's mirror image,
as the reference's counter pulse of phi = pi) on a hydrogen blob of
1e-2 n_cr in a sphere of 2 lambda radius at the centre, 4 particles per cell
of electrons and protons, dx = lambda/32, dt = 0.3 dx (the five-point scheme
needs dt below about 0.35 dx on cubic cells).  The state is generated on the
GPU (seeded); positrons and photons start empty.

The cascade multiplies the particles about tenfold every 50 steps at this
field; as the reference does in such runs, particle merging bounds them:
after a step in which a species holds more than crpc macro-particles per
cell, that species is thinned by the reference's "nl" merging
(evaluate_merging_condition / pmerging, main.cpp:1691-1748, mc.cpp:198-462:
deletion probability (n - crpc cells) / n weighted by the particle's charge,
survivors' weights raised so that the species' charge is kept) before the
next step.

Prints, every `--every` steps, the macro-particles per species and the
elapsed time (CUDA events on the stream, host work between steps included),
and at the end one JSON line: particle-steps/s over the whole run (the
particles pushed in each step, summed, over that time, merging included),
the final counts, the peak particle count, and the mean time per step of
each phase (`ms_per_step`; push_deposit contains qed_prepare, the push
kernels and the born-count read-back, which are also given apart; merging
is averaged over all steps).
"""
from __future__ import annotations

import argparse
import json
import time


def reservation(nc: int, crpc: float, n_ions: int) -> list[int]:
    """Particle slots to reserve per species (electrons, protons, positrons,
    photons) so that the cascade never grows a store mid-run.

    Merging keeps each species near crpc * nc macro-particles between steps.
    Before each QED push the library needs, in the worst case, one new pair
    per photon in each lepton store and one new photon per lepton in the
    photon store; the photons are bounded by the same merging.  Four times
    the merging bound per lepton store and six times for the photons covers
    both with room for a step's growth above the bound."""
    crnp = int(crpc * nc)
    return [4 * crnp, n_ions + 1024, 4 * crnp, 6 * crnp]


def run(grid=(256, 256, 256), steps=600, precision="fp64", seed=0, every=50, crpc=1.5, device=0, quiet=False,
        reserve=True):
    import torch

    from . import workloads as W
    from .api import Region

    case = W.config("cfg3_256_fivepoint_vay_qed")
    if tuple(grid) != (case.nx, case.ny, case.nz):
        case = W.scaled(case, *grid)
    case.seed = seed
    dev = f"cuda:{device}"
    torch.cuda.set_device(device)
    stream = torch.cuda.Stream(device=device)
    torch.cuda.set_stream(stream)
    species = (-1.0, W.PROTON_CMR, 1.0, 0.0)  # electrons, protons, positrons, photons
    n_ions = sum(ch["x"].numel() for ch in W.particle_chunks_torch(case, case.species[1], 32, device=dev,
                                                                     seed=seed + 17))
    capacity = reservation(case.nx * case.ny * case.nz, crpc, n_ions) if reserve else None
    reg = Region(case.nx, case.ny, case.nz, case.dx, case.dx, case.dx, case.dt, species_cmr=species,
                 solver=case.solver, pusher=case.pusher, qed=True, precision=precision, seed=seed,
                 capacity=capacity, device=device)
    reg.set_stream(stream.cuda_stream)
    reg.set_timing(True)
    f = W.make_fields_torch(case, device=dev)
    torch.cuda.synchronize()
    import ctypes as C
    ptr = lambda t: C.cast(t.data_ptr(), C.POINTER(C.c_double))
    reg._check(reg.lib.qp_load_fields(reg.h, *[ptr(f[k]) for k in ("ex", "ey", "ez", "bx", "by", "bz")]))
    del f
    reg.init_boundaries()
    keys = ("x", "y", "z", "ux", "uy", "uz", "g", "q")
    for si, sp in enumerate(case.species):
        for ch in W.particle_chunks_torch(case, sp, 32, device=dev, seed=seed + 17 * si):
            reg._check(reg.lib.qp_load_particles(reg.h, si, ch["x"].numel(), *[ptr(ch[k]) for k in keys], None))
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    counts = [reg.count(i) for i in range(len(species))]
    n0 = sum(counts)
    if not quiet:
        print(f"{case.nx}x{case.ny}x{case.nz} cells, {precision}, start: {counts} (e, p+, e+, photons)", flush=True)
    pushed, peak, ms_total, merges = 0, n0, 0.0, 0
    merge_events = []
    history = []
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    crnp = crpc * case.nx * case.ny * case.nz
    t_wall = time.perf_counter()
    counts = [reg.count(i) for i in range(len(species))]
    e0.record(stream)
    for step in range(1, steps + 1):
        pushed += sum(counts)
        d = reg.step(1)[0]
        counts = [int(d.n_macro[i]) for i in range(len(species))]
        peak = max(peak, sum(counts))
        # the nl merging condition per species (main.cpp:1691-1748)
        ppd = [(n - crnp) / n if n > crnp else 0.0 for n in counts]
        if any(v > 0 for v in ppd):
            m0, m1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            m0.record(stream)
            reg.pmerging("nl", ppd)
            m1.record(stream)
            merge_events.append((m0, m1))
            merges += 1
            counts = [reg.count(i) for i in range(len(species))]
        if step % every == 0 or step == steps:
            e1.record(stream)
            e1.synchronize()
            ms_total = e0.elapsed_time(e1)
            history.append({"step": step, "counts": counts, "ms": ms_total, "merges": merges})
            if not quiet:
                print(f"step {step}: {counts}, {sum(counts):.3e} particles, {ms_total / 1e3:.2f} s, "
                      f"{merges} merging passes", flush=True)
    phase, nph = reg.get_timing()
    merge_ms = sum(a.elapsed_time(b) for a, b in merge_events)
    qed, nq = reg.get_qed_timing()
    reg.close()
    per = lambda v, n: float(v) / max(n, 1)
    return {"metric": "QED particle-steps/s", "value": pushed / (ms_total * 1e-3), "unit": "particle-steps/s",
            "precision": precision, "grid": list(grid), "steps": steps, "seconds_device": ms_total / 1e3,
            "seconds_wall": time.perf_counter() - t_wall, "particles_start": n0, "particles_end": sum(counts),
            "particles_peak": peak, "counts_end": counts, "merging_passes": merges, "crpc": crpc,
            "reserved_slots": capacity,
            "ms_per_step": {"push_deposit": per(phase[0], nph), "rebin": per(phase[1], nph),
                            "fields": per(phase[2], nph), "diag": per(phase[3], nph),
                            "qed_prepare": per(qed[0], nq), "push_kernels": per(qed[1], nq),
                            "born_readback": per(qed[2], nq), "merging": merge_ms / max(steps, 1)},
            "history": history}


def _main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--grid", type=int, nargs=3, default=(256, 256, 256))
    ap.add_argument("--steps", type=int, default=600)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--every", type=int, default=50)
    ap.add_argument("--crpc", type=float, default=1.5,
                    help="macro-particles per cell above which a species is merged")
    ap.add_argument("--no-reserve", action="store_true",
                    help="let the stores grow on demand instead of reserving them up front")
    a = ap.parse_args()
    r = run(tuple(a.grid), a.steps, a.precision, a.seed, a.every, a.crpc, reserve=not a.no_reserve)
    print(json.dumps(r), flush=True)


if __name__ == "__main__":
    _main()
