"""ctypes binding of libquill_b200.so (the C ABI in include/quill_b200.h).

`Region` mirrors the reference's step contract on `spatial_region`
(include/main.h:17-170): load fields and particles, `init_boundaries`
(f_init_boundaries + interpolate_be), `step` (birth_from_vacuum -> padvance
-> compute_N / compute_energy -> fadvance, main.cpp:2321-2331), and dumps.

There is no CPU fallback: constructing a Region without the built library
or without a CUDA device raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libquill_b200.so")

QP_MAX_SPECIES = 8
SOLVERS = {"fdtd": 0, "ndfx": 1, "five_point": 2}
PUSHERS = {"vay": 0, "boris": 1}
PRECISIONS = {"fp64": 0, "mixed": 1}
STATUS = {0: "QP_OK", 1: "QP_ERR_CONFIG", 2: "QP_ERR_CAPACITY", 3: "QP_ERR_NAN", 4: "QP_ERR_TIMEOUT",
          5: "QP_ERR_CUDA", 6: "QP_ERR_STATE", 7: "QP_ERR_ARG"}


class QPError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


class Params(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double), ("dt", C.c_double),
        ("lambda_cm", C.c_double),
        ("solver", C.c_int), ("pusher", C.c_int), ("qed", C.c_int), ("precision", C.c_int),
        ("seed", C.c_uint64),
        ("n_species", C.c_int),
        ("cmr", C.c_double * QP_MAX_SPECIES),
        ("capacity", C.c_int64 * QP_MAX_SPECIES),
        ("device", C.c_int),
    ]


class Diag(C.Structure):
    _fields_ = [
        ("N_e", C.c_double), ("N_p", C.c_double), ("N_ph", C.c_double),
        ("N_qp_e", C.c_int64), ("N_qp_p", C.c_int64), ("N_qp_g", C.c_int64),
        ("energy_f", C.c_double), ("energy_e", C.c_double), ("energy_p", C.c_double),
        ("energy_ph", C.c_double),
        ("n_ion", C.c_int),
        ("N_qp_i", C.c_int64 * QP_MAX_SPECIES),
        ("ienergy", C.c_double * QP_MAX_SPECIES),
        ("n_macro", C.c_int64 * QP_MAX_SPECIES),
        ("status", C.c_int32), ("pad_", C.c_int32),
        ("energy_erased", C.c_double),
        ("energy_erased_sp", C.c_double * QP_MAX_SPECIES),
    ]

    def total_energy(self) -> float:
        """Fields + electrons + positrons + photons + ions (the sum of the
        `energy` output's columns)."""
        return (self.energy_f + self.energy_e + self.energy_p + self.energy_ph
                + sum(self.ienergy[m] for m in range(self.n_ion)))

    def as_array(self) -> np.ndarray:
        """Same layout as the CPU checkers' diagnostic rows: N_e N_p N_ph
        N_qp_e N_qp_p N_qp_g energy_f energy_e energy_p energy_ph, then
        (N_qp_i, ienergy) per ion population."""
        v = [self.N_e, self.N_p, self.N_ph, self.N_qp_e, self.N_qp_p, self.N_qp_g,
             self.energy_f, self.energy_e, self.energy_p, self.energy_ph]
        for m in range(self.n_ion):
            v += [self.N_qp_i[m], self.ienergy[m]]
        return np.array(v, dtype=np.float64)


_lib = None


def load_library(path: str | None = None):
    """Load libquill_b200.so; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise ImportError(f"libquill_b200.so not built at {p}: run `python -m quill_b200.build`")
    lib = C.CDLL(p)
    D, DP, I64, I64P, VP = C.c_double, C.POINTER(C.c_double), C.c_int64, C.POINTER(C.c_int64), C.c_void_p
    sig = {
        "qp_version": (C.c_char_p, []),
        "qp_last_error": (C.c_char_p, [VP]),
        "qp_create": (C.c_int, [C.POINTER(Params), C.POINTER(VP)]),
        "qp_destroy": (C.c_int, [VP]),
        "qp_load_fields": (C.c_int, [VP] + [DP] * 6),
        "qp_init_boundaries": (C.c_int, [VP]),
        "qp_load_particles": (C.c_int, [VP, C.c_int, I64] + [DP] * 9),
        "qp_step": (C.c_int, [VP, C.c_int, D, C.POINTER(Diag)]),
        "qp_get_diag": (C.c_int, [VP, C.POINTER(Diag)]),
        "qp_dump_fields": (C.c_int, [VP, DP]),
        "qp_count_particles": (C.c_int, [VP, C.c_int, I64P]),
        "qp_dump_particles": (C.c_int, [VP, C.c_int, I64] + [DP] * 9 + [I64P]),
        "qp_checkpoint": (C.c_int, [VP, C.c_int]),
        "qp_restore": (C.c_int, [VP, C.c_int]),
        "qp_synchronize": (C.c_int, [VP]),
        "qp_set_stream": (C.c_int, [VP, VP]),
        "qp_launch_count": (C.c_int, [VP, I64P]),
        "qp_set_timing": (C.c_int, [VP, C.c_int]),
        "qp_eval_qed_rates": (C.c_int, [C.c_int, D, I64, DP, DP]),
        "qp_eval_qed_rates_noalloc": (C.c_int, [C.c_int, D, I64, DP, DP]),
        "qp_get_timing": (C.c_int, [VP, DP, I64P]),
        "qp_get_qed_timing": (C.c_int, [VP, DP, I64P]),
        "qp_set_erased_tracking": (C.c_int, [VP, C.c_int]),
        "qp_set_ordered_current": (C.c_int, [VP, C.c_int]),
        "qp_pmerging": (C.c_int, [VP, C.c_int, DP]),
        "qp_moving_window": (C.c_int, [VP]),
        "qp_set_catching": (C.c_int, [VP, C.c_int, I64]),
        "qp_set_dump_photons": (C.c_int, [VP, C.c_int, I64]),
        "qp_set_tracking": (C.c_int, [VP, C.c_int]),
        "qp_set_diag_range": (C.c_int, [VP, C.c_int, C.c_int]),
        "qp_get_field_slab": (C.c_int, [VP, C.c_int, C.c_int, DP]),
        "qp_set_field_slab": (C.c_int, [VP, C.c_int, C.c_int, DP]),
        "qp_get_particle_slab": (C.c_int, [VP, C.c_int, C.c_int, C.c_int, I64] + [DP] * 9 + [I64P]),
        "qp_replace_particle_slab": (C.c_int, [VP, C.c_int, C.c_int, C.c_int, I64] + [DP] * 9),
        "qp_layer_counts": (C.c_int, [VP, I64P]),
        "qp_max_w": (C.c_int, [VP, C.c_int, C.c_int, DP]),
        "qp_dump_field_slices": (C.c_int, [VP, C.c_int, DP]),
        "qp_first_in_cells": (C.c_int, [VP, C.c_int, I64, I64P, I64P]),
        "qp_set_track_numbers": (C.c_int, [VP, C.c_int, I64, I64P, I64P]),
        "qp_get_tracked": (C.c_int, [VP, C.c_int, I64, I64P] + [DP] * 9 + [I64P]),
        "qp_get_caught": (C.c_int, [VP, I64, C.POINTER(C.c_int32)] + [DP] * 9 + [I64P, I64P]),
        "qp_adjoint_energy": (C.c_int, [VP, C.c_int, C.c_int, D, DP, DP, DP]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def _dp(a):
    """double* of a numpy array, or of a torch tensor (host or device: the
    entry points that take it copy with cudaMemcpyDefault)."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        if str(a.dtype) != "torch.float64" or not a.is_contiguous():
            raise ValueError("tensor arguments must be contiguous float64")
        return C.cast(C.c_void_p(a.data_ptr()), C.POINTER(C.c_double))
    return a.ctypes.data_as(C.POINTER(C.c_double))


PARTICLE_KEYS = ("x", "y", "z", "ux", "uy", "uz", "g", "q", "chi")


def eval_qed_rates(samples: np.ndarray, lambda_cm: float = 1e-4, device: int = 0) -> np.ndarray:
    """Device evaluation of chi, w, r-after-w, tilde_w, vacuum W for rows of
    (e[3] b[3] u[3] g r chi)."""
    lib = load_library()
    a = np.ascontiguousarray(samples, dtype=np.float64).reshape(-1, 12)
    out = np.zeros((a.shape[0], 5))
    r = lib.qp_eval_qed_rates(device, lambda_cm, a.shape[0], _dp(a), _dp(out))
    if r != 0:
        raise QPError(r, lib.qp_last_error(None).decode())
    return out


class Region:
    """One simulation region on one GPU."""

    def __init__(self, nx, ny, nz, dx, dy, dz, dt, *, species_cmr=(-1.0,), lambda_cm=1e-4,
                 solver="fdtd", pusher="boris", qed=False, precision="fp64", seed=0,
                 capacity=None, device=0):
        lib = load_library()
        self.lib = lib
        p = Params()
        p.nx, p.ny, p.nz = nx, ny, nz
        p.dx, p.dy, p.dz, p.dt = dx, dy, dz, dt
        p.lambda_cm = lambda_cm
        p.solver = SOLVERS[solver] if isinstance(solver, str) else int(solver)
        p.pusher = PUSHERS[pusher] if isinstance(pusher, str) else int(pusher)
        p.qed = int(bool(qed))
        p.precision = PRECISIONS[precision] if isinstance(precision, str) else int(precision)
        p.seed = seed
        p.n_species = len(species_cmr)
        for i, c in enumerate(species_cmr):
            p.cmr[i] = c
            p.capacity[i] = int(capacity[i]) if capacity is not None else 0
        p.device = device
        h = C.c_void_p()
        r = lib.qp_create(C.byref(p), C.byref(h))
        if r != 0:
            raise QPError(r, lib.qp_last_error(None).decode())
        self.h = h
        self.params = p
        self.shape = (nx, ny, nz)
        self.n_species = len(species_cmr)

    def _check(self, r):
        if r != 0:
            raise QPError(r, self.lib.qp_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.qp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def nc(self):
        nx, ny, nz = self.shape
        return nx * ny * nz

    def set_fields(self, ex, ey, ez, bx, by, bz):
        arrs = [np.ascontiguousarray(a, dtype=np.float64).reshape(-1) for a in (ex, ey, ez, bx, by, bz)]
        for a in arrs:
            if a.size != self.nc:
                raise ValueError("field plane size mismatch")
        self._check(self.lib.qp_load_fields(self.h, *[_dp(a) for a in arrs]))

    def init_boundaries(self):
        self._check(self.lib.qp_init_boundaries(self.h))

    def add_particles(self, species: int, parts: dict):
        n = len(parts["x"])
        arrs = []
        for k in PARTICLE_KEYS:
            a = parts.get(k)
            arrs.append(None if a is None else np.ascontiguousarray(a, dtype=np.float64))
        self._check(self.lib.qp_load_particles(self.h, species, n, *[_dp(a) for a in arrs]))

    def step(self, nsteps=1, external_bz=0.0) -> list:
        d = (Diag * max(nsteps, 1))()
        self._check(self.lib.qp_step(self.h, nsteps, external_bz, d))
        return [d[i] for i in range(nsteps)]

    def get_diag(self) -> Diag:
        d = Diag()
        self._check(self.lib.qp_get_diag(self.h, C.byref(d)))
        return d

    def get_fields(self) -> np.ndarray:
        out = np.empty((12,) + self.shape, dtype=np.float64)
        self._check(self.lib.qp_dump_fields(self.h, _dp(out)))
        return out

    def count(self, species: int) -> int:
        n = C.c_int64()
        self._check(self.lib.qp_count_particles(self.h, species, C.byref(n)))
        return n.value

    def get_particles(self, species: int) -> dict:
        n = self.count(species)
        cap = max(n, 1)
        out = {k: np.zeros(cap) for k in PARTICLE_KEYS}
        cell = np.zeros(cap, dtype=np.int64)
        self._check(self.lib.qp_dump_particles(self.h, species, cap, *[_dp(out[k]) for k in PARTICLE_KEYS],
                                               cell.ctypes.data_as(C.POINTER(C.c_int64))))
        d = {k: v[:n] for k, v in out.items()}
        d["cell"] = cell[:n]
        return d

    def checkpoint(self, slot=0):
        self._check(self.lib.qp_checkpoint(self.h, slot))

    def restore(self, slot=0):
        self._check(self.lib.qp_restore(self.h, slot))

    def synchronize(self):
        self._check(self.lib.qp_synchronize(self.h))

    def set_stream(self, stream_ptr: int):
        self._check(self.lib.qp_set_stream(self.h, C.c_void_p(stream_ptr)))

    def set_diag_range(self, i_lo: int, i_hi: int):
        self._check(self.lib.qp_set_diag_range(self.h, int(i_lo), int(i_hi)))

    def layer_counts(self) -> np.ndarray:
        """Quasiparticles per x-layer, all species."""
        out = np.zeros(self.shape[0], dtype=np.int64)
        self._check(self.lib.qp_layer_counts(self.h, out.ctypes.data_as(C.POINTER(C.c_int64))))
        return out

    def field_slices(self, ix: int) -> np.ndarray:
        """(12, nx*(ny+nz) + ny*nz): the output slices of each field plane."""
        nx, ny, nz = self.shape
        out = np.zeros((12, nx * (ny + nz) + ny * nz))
        self._check(self.lib.qp_dump_field_slices(self.h, ix, _dp(out)))
        return out

    def max_w(self, i0: int = 0, i1: int | None = None) -> float:
        """max of E^2 + B^2 over the cells with i in [i0, i1)."""
        v = C.c_double()
        self._check(self.lib.qp_max_w(self.h, i0, self.shape[0] if i1 is None else i1, C.byref(v)))
        return v.value

    # one slab exchange per species
    @property
    def species_ids(self):
        return tuple(range(self.n_species))

    def get_field_slab(self, i0: int, width: int, out=None):
        """E B J Bbar of the cells with i in [i0, i0 + width): (12, width,
        ny, nz) float64, into `out` (numpy or torch, host or device) if given."""
        if out is None:
            out = np.zeros((12, width, self.shape[1], self.shape[2]))
        self._check(self.lib.qp_get_field_slab(self.h, i0, width, _dp(out)))
        return out

    def set_field_slab(self, i0: int, planes12):
        a = planes12 if hasattr(planes12, "data_ptr") else np.ascontiguousarray(planes12, dtype=np.float64)
        width = a.numel() // (12 * self.shape[1] * self.shape[2]) if hasattr(a, "numel") else \
            a.size // (12 * self.shape[1] * self.shape[2])
        self._check(self.lib.qp_set_field_slab(self.h, i0, width, _dp(a)))

    def get_particle_slab(self, species: int, i0: int, width: int, device=None) -> dict:
        """The species' particles in the slab, in traversal order: numpy
        arrays, or torch float64 tensors on `device` if given."""
        n = C.c_int64()
        self._check(self.lib.qp_get_particle_slab(self.h, species, i0, width, 0, *([None] * 9), C.byref(n)))
        m = n.value
        if device is not None:
            import torch
            buf = torch.empty((len(PARTICLE_KEYS), max(m, 1)), dtype=torch.float64, device=device)
        else:
            buf = np.zeros((len(PARTICLE_KEYS), max(m, 1)))
        if m:
            rows = [buf[i] for i in range(len(PARTICLE_KEYS))]
            self._check(self.lib.qp_get_particle_slab(self.h, species, i0, width, m, *[_dp(r) for r in rows],
                                                      C.byref(n)))
        return {k: buf[i, :m] for i, k in enumerate(PARTICLE_KEYS)}

    def replace_particle_slab(self, species: int, i0: int, width: int, parts: dict):
        """Replace the species' particles in the slab by `parts` (numpy or
        torch arrays; in the given order inside each cell)."""
        n = len(parts["x"])
        arrs = []
        for k in PARTICLE_KEYS:
            a = parts.get(k)
            if a is None:
                arrs.append(None)
            elif hasattr(a, "data_ptr"):
                arrs.append(a.contiguous())
            else:
                arrs.append(np.ascontiguousarray(a, dtype=np.float64))
        self._check(self.lib.qp_replace_particle_slab(self.h, species, i0, width, n, *[_dp(a) for a in arrs]))

    def set_tracking(self, enable: bool = True):
        self._check(self.lib.qp_set_tracking(self.h, int(bool(enable))))

    def first_in_cells(self, species: int, cells) -> np.ndarray:
        c = np.ascontiguousarray(np.asarray(cells, dtype=np.int64))
        out = np.zeros(max(c.size, 1), dtype=np.int64)
        lp = C.POINTER(C.c_int64)
        self._check(self.lib.qp_first_in_cells(self.h, species, c.size, c.ctypes.data_as(lp), out.ctypes.data_as(lp)))
        return out[:c.size]

    def set_track_numbers(self, species: int, positions, numbers):
        p = np.ascontiguousarray(np.asarray(positions, dtype=np.int64))
        nn = np.ascontiguousarray(np.asarray(numbers, dtype=np.int64))
        lp = C.POINTER(C.c_int64)
        self._check(self.lib.qp_set_track_numbers(self.h, species, p.size, p.ctypes.data_as(lp), nn.ctypes.data_as(lp)))

    def get_tracked(self, species: int) -> dict:
        n = C.c_int64()
        lp = C.POINTER(C.c_int64)
        self._check(self.lib.qp_get_tracked(self.h, species, 0, None, *([None] * 9), C.byref(n)))
        m = max(n.value, 1)
        trn = np.zeros(m, dtype=np.int64)
        arrs = {k: np.zeros(m) for k in ("x", "y", "z", "ux", "uy", "uz", "g", "q", "chi")}
        self._check(self.lib.qp_get_tracked(self.h, species, m, trn.ctypes.data_as(lp),
                                            *[_dp(arrs[k]) for k in ("x", "y", "z", "ux", "uy", "uz", "g", "q", "chi")],
                                            C.byref(n)))
        out = {k: v[:n.value] for k, v in arrs.items()}
        out["trn"] = trn[:n.value]
        return out

    def set_catching(self, enable: bool = True, capacity: int = 1 << 20):
        """Record the particles the steps erase (catching)."""
        self._check(self.lib.qp_set_catching(self.h, int(bool(enable)), int(capacity)))

    def set_dump_photons(self, enable: bool = True, capacity: int = 1 << 20):
        self._check(self.lib.qp_set_dump_photons(self.h, int(bool(enable)), int(capacity)))

    def get_caught(self) -> dict:
        """The recorded particles (empties the buffer): species, x y z (cell
        units), ux uy uz g q chi, and the number dropped for lack of room."""
        n, dropped = C.c_int64(), C.c_int64()
        null = [None] * 9
        self._check(self.lib.qp_get_caught(self.h, 0, None, *null, C.byref(n), C.byref(dropped)))
        m = max(n.value, 1)
        sp = np.zeros(m, dtype=np.int32)
        arrs = {k: np.zeros(m) for k in ("x", "y", "z", "ux", "uy", "uz", "g", "q", "chi")}
        self._check(self.lib.qp_get_caught(self.h, m, sp.ctypes.data_as(C.POINTER(C.c_int32)),
                                           *[_dp(arrs[k]) for k in ("x", "y", "z", "ux", "uy", "uz", "g", "q", "chi")],
                                           C.byref(n), C.byref(dropped)))
        out = {k: v[:n.value] for k, v in arrs.items()}
        out["species"] = sp[:n.value]
        out["dropped"] = dropped.value
        return out

    def moving_window(self):
        """Shift the region one cell towards -x (spatial_region::moving_window)."""
        self._check(self.lib.qp_moving_window(self.h))

    def pmerging(self, mode: str, ppd):
        """Particle merging ("ti" or "nl"); ppd per species in table order
        ("ti" uses ppd[0] for all)."""
        p = np.zeros(self.n_species)
        v = np.asarray(ppd, dtype=np.float64).reshape(-1)
        p[:min(v.size, p.size)] = v[:p.size]
        self._check(self.lib.qp_pmerging(self.h, 1 if mode == "ti" else 2, _dp(p)))

    def set_erased_tracking(self, enable: bool = True):
        """Report in Diag.energy_erased the energy of the particles each step
        erases (QED-off steps)."""
        self._check(self.lib.qp_set_erased_tracking(self.h, int(bool(enable))))

    def set_ordered_current(self, enable: bool = True):
        """Sum J in the reference's order (FP64, QED off): the region then
        stays bit-identical to the reference over any number of steps."""
        self._check(self.lib.qp_set_ordered_current(self.h, int(bool(enable))))

    def set_timing(self, enable: bool = True):
        self._check(self.lib.qp_set_timing(self.h, int(bool(enable))))

    def get_timing(self):
        """(ms per phase [push, rebin, fields, diag], steps timed)."""
        ms = np.zeros(4)
        n = C.c_int64()
        self._check(self.lib.qp_get_timing(self.h, _dp(ms), C.byref(n)))
        return ms, n.value

    def get_qed_timing(self):
        """(ms [preparation incl. vacuum pairs and one host sync, push
        kernels, born-count read-back], QED steps timed)."""
        ms = np.zeros(3)
        n = C.c_int64()
        self._check(self.lib.qp_get_qed_timing(self.h, _dp(ms), C.byref(n)))
        return ms, n.value

    def adjoint_energy(self, nsteps: int, every: int = 32, external_bz: float = 0.0):
        """Run nsteps steps from the current state and return (L, dL/dfields,
        dL/dq): L = energy_e after the last step, dL/dfields of shape
        (6, nx, ny, nz) for the planes as loaded (Ex Ey Ez Bx By Bz), dL/dq per
        particle of species 0 in its traversal order at entry.  The region is
        left in its state at entry."""
        n = self.count(0)
        gf = np.zeros((6,) + self.shape)
        gq = np.zeros(max(n, 1))
        loss = C.c_double()
        self._check(self.lib.qp_adjoint_energy(self.h, nsteps, every, external_bz, _dp(gf), _dp(gq),
                                               C.byref(loss)))
        return loss.value, gf, gq[:n]

    def launch_count(self) -> int:
        n = C.c_int64()
        self._check(self.lib.qp_launch_count(self.h, C.byref(n)))
        return n.value
