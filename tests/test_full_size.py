"""The 512^3 benchmark configuration at its full size (1.34e8 cells, 5.25e8
electrons, FDTD + Boris, 4 ppc at 0.05 n_cr, 10 keV, laser a0 = 20), checked
through properties that do not depend on the size, since the CPU checker
cannot step this box:

* charge conservation: the discrete Gauss residual
  R = (Ex[i] - Ex[i-1]) + (Ey[j] - Ey[j-1]) + (Ez[k] - Ez[k-1]) - dx * rho
  (rho: cloud-in-cell charge of the particles at the nodes) does not change
  at interior nodes over the steps (the Yee curl has zero discrete
  divergence and the 12-term segment deposition of deposition.cpp:13-356
  satisfies the discrete continuity equation).  Particles erased by
  p_boundary sit in the layers {0, n-2, n-1}, whose nodes are excluded;
* the traversal order: the cells of the particles, read slab by slab in
  traversal order, never decrease;
* the particle count: the slabs hold every particle of the store, and the
  step's diagnostics count them (compute_N, fout.cpp:41-85).

Both precisions, two steps each; about 90 GB of device memory in FP64.
"""
import ctypes as C

import pytest

from tests.conftest import gpu_available

SLAB = 32  # x-layers read at a time


def _build(precision, n=None):
    import torch

    from quill_b200 import workloads as W
    from quill_b200.api import Region
    case = W.config("cfg5_512_fdtd_boris")
    if n is not None:
        case = W.scaled(case, n, n, n)
    dev = "cuda:0"
    # one stream for torch and the library (the library's own stream is not
    # ordered with torch's legacy default stream)
    torch.cuda.set_stream(torch.cuda.Stream(device=dev))
    f = W.make_fields_torch(case, device=dev)
    reg = Region(case.nx, case.ny, case.nz, case.dx, case.dx, case.dx, case.dt,
                 species_cmr=tuple(sp.cmr for sp in case.species), solver=case.solver, pusher=case.pusher,
                 precision=precision, device=0)
    reg.set_stream(torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    ptr = lambda t: C.cast(t.data_ptr(), C.POINTER(C.c_double))
    reg._check(reg.lib.qp_load_fields(reg.h, *[ptr(f[k]) for k in ("ex", "ey", "ez", "bx", "by", "bz")]))
    del f
    reg.init_boundaries()
    keys = ("x", "y", "z", "ux", "uy", "uz", "g", "q")
    for ch in W.particle_chunks_torch(case, case.species[0], 48, device=dev, seed=case.seed):
        reg._check(reg.lib.qp_load_particles(reg.h, 0, ch["x"].numel(), *[ptr(ch[k]) for k in keys], None))
        del ch
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    return case, reg


def _residual(case, reg):
    """(R at the interior nodes, max |dx rho|, max |E|, particles read, cells
    ordered)."""
    import torch
    nx, ny, nz = case.nx, case.ny, case.nz
    dev = "cuda:0"
    rho = torch.zeros((nx, ny, nz), dtype=torch.float64, device=dev)
    flat = rho.view(-1)
    total, ordered, last = 0, True, -1
    for i0 in range(0, nx, SLAB):
        w = min(SLAB, nx - i0)
        p = reg.get_particle_slab(0, i0, w, device=dev)
        n = p["x"].numel()
        if n == 0:
            continue
        total += n
        ii, jj, kk = (torch.floor(p[a]).to(torch.int64) for a in ("x", "y", "z"))
        # every particle lies in a cell whose +1 corner node is in the box
        # (checked here, on the host, before any index is used on the device)
        for name, v, hi in (("i", ii, nx - 1), ("j", jj, ny - 1), ("k", kk, nz - 1)):
            lo_v, hi_v = (int(t) for t in torch.aminmax(v))
            assert 0 <= lo_v and hi_v < hi, f"slab {i0}: {name} cells in [{lo_v}, {hi_v}]"
        cell = (ii * ny + jj) * nz + kk
        ordered &= bool((cell[1:] >= cell[:-1]).all()) and int(cell[0]) >= last
        last = int(cell[-1])
        fx, fy, fz = p["x"] - ii, p["y"] - jj, p["z"] - kk
        q = p["q"]
        del p
        for di, wx in ((0, 1 - fx), (1, fx)):
            for dj, wy in ((0, 1 - fy), (1, fy)):
                for dk, wz in ((0, 1 - fz), (1, fz)):
                    flat.index_add_(0, ((ii + di) * ny + jj + dj) * nz + kk + dk, q * wx * wy * wz)
        del ii, jj, kk, cell, fx, fy, fz, q
    div = torch.zeros_like(rho)
    e12 = torch.empty((12, nx, ny, nz), dtype=torch.float64, device=dev)
    reg.get_field_slab(0, nx, out=e12)
    ex, ey, ez = e12[0], e12[1], e12[2]
    emax = float(e12[:3].abs().max())
    div[1:] += ex[1:] - ex[:-1]
    div[:, 1:] += ey[:, 1:] - ey[:, :-1]
    div[:, :, 1:] += ez[:, :, 1:] - ez[:, :, :-1]
    del e12, ex, ey, ez
    div -= case.dx * rho
    scale = float((case.dx * rho).abs().max())
    del rho
    s = slice(2, -2)
    r = div[s, s, s].clone()
    del div
    torch.cuda.empty_cache()
    return r, scale, emax, total, ordered


@pytest.mark.gpu
@pytest.mark.parametrize("precision,n", [("fp64", 96), ("fp64", None), ("mixed", None)])
def test_full_size_charge_order_count(precision, n):
    """n = None: the full 512^3 box; 96: the same physics on 96^3 first."""
    if not gpu_available():
        pytest.skip("needs a CUDA device")
    import torch
    case, reg = _build(precision, n)
    try:
        n0 = reg.count(0)
        r0, scale, emax, total0, ordered0 = _residual(case, reg)
        assert total0 == n0 and ordered0
        d = reg.step(2)
        n1 = reg.count(0)
        r1, _, _, total1, ordered1 = _residual(case, reg)
        assert total1 == n1, (total1, n1)
        assert ordered1, "cells out of traversal order after the steps"
        assert int(d[-1].n_macro[0]) == n1
        assert 0.99 * n0 < n1 <= n0  # thermal particles leave through the absorbing layers only
        dr = float((r1 - r0).abs().max())
        print(f"{precision} {case.nx}^3: {n0} -> {n1} particles, max |dR| = {dr:.3e}, "
              f"max |dx rho| = {scale:.3e}, max |E| = {emax:.3e}")
        if precision == "fp64":
            # FP64 round-off (the J sums' order differs from the reference's)
            assert dr < 1e-12 * scale, f"Gauss residual changed by {dr / scale:.3e} of max |dx rho|"
        else:
            # FP32 round-off of the E updates: about an ulp of the largest E
            # (the laser, |E| ~ 20 here) per step; one misplaced current term
            # (q d ~ 1e-3) would exceed this bound
            bound = 1e-5 * max(scale, emax)
            assert dr < bound, f"Gauss residual changed by {dr:.3e} (bound {bound:.3e})"
    finally:
        reg.close()
        torch.cuda.synchronize()
        torch.cuda.set_stream(torch.cuda.default_stream())
        torch.cuda.empty_cache()
