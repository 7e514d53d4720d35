"""ORACLE / TEST INFRASTRUCTURE — ctypes loader for the CPU checkers.

Two interchangeable back ends with one interface:

* ``kind="ref"``  — the reference's own sources (QUILL src/*.cpp minus
  main.cpp) compiled with oracle/ref_shim.cpp into oracle/_ref/ by
  ``make -C oracle ref``;
* ``kind="port"`` — the plain-C restatement oracle/qp_oracle.c built by
  ``make -C oracle``.

Each comes in a ``parity`` flavour (-ffp-contract=off: plain IEEE operation
sequence, comparable bit for bit with the CUDA FP64 path built with
--fmad=false) and a ``fast`` flavour (Release flags, for CPU timing).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module, and only to check or time against it.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

_D = C.c_double
_DP = C.POINTER(C.c_double)
_LP = C.POINTER(C.c_long)


def _has_avx512() -> bool:
    try:
        with open("/proc/cpuinfo") as f:
            flags = f.read()
        return " avx512f " in flags and " avx512vl " in flags and " avx512_fp16 " in flags
    except OSError:
        return False


def lib_path(kind: str = "port", flavour: str = "parity") -> str:
    if flavour == "fast" and _has_avx512():
        v4 = lib_path(kind, "fast_v4")
        if os.path.exists(v4):
            return v4
    if kind == "ref":
        return os.path.join(HERE, "_ref", f"libquill_ref_{flavour}.so")
    return os.path.join(HERE, f"liboracle_{flavour}.so")


def available(kind: str = "port", flavour: str = "parity") -> bool:
    return os.path.exists(lib_path(kind, flavour))


_LIBS: dict = {}


def _load(kind: str, flavour: str):
    key = (kind, flavour)
    if key in _LIBS:
        return _LIBS[key]
    path = lib_path(kind, flavour)
    if not os.path.exists(path):
        raise FileNotFoundError(f"oracle library missing: {path} (run `make -C oracle{' ref' if kind == 'ref' else ''}`)")
    lib = C.CDLL(path)
    p = "qref_" if kind == "ref" else "qor_"

    def fn(name, res, *args):
        f = getattr(lib, p + name)
        f.restype = res
        f.argtypes = list(args)
        return f

    api = {
        "create": fn("create", C.c_void_p, C.c_int, C.c_int, C.c_int, _D, _D, _D, _D, _D,
                     C.c_int, C.c_int, C.c_int, C.c_int, _DP, C.c_int),
        "destroy": fn("destroy", None, C.c_void_p),
        "set_fields": fn("set_fields", None, C.c_void_p, _DP, _DP, _DP, _DP, _DP, _DP),
        "get_fields": fn("get_fields", None, C.c_void_p, _DP),
        "init_boundaries": fn("init_boundaries", None, C.c_void_p),
        "add_particles": fn("add_particles", None, C.c_void_p, C.c_long, _DP, _DP, _DP, _DP, _DP,
                            _DP, _DP, _DP, _DP, _DP),
        "count_particles": fn("count_particles", C.c_long, C.c_void_p),
        "get_particles": fn("get_particles", C.c_long, C.c_void_p, C.c_long, _DP, _LP),
        "diag_len": fn("diag_len", C.c_int, C.c_void_p),
        "step": fn("step", None, C.c_void_p, C.c_int, _D, _DP),
        "padvance": fn("padvance", None, C.c_void_p, _D),
        "fadvance": fn("fadvance", None, C.c_void_p),
        "compute_diag": fn("compute_diag", None, C.c_void_p, _DP),
        "push": fn("push", None, C.c_int, _D, _DP, _DP, _DP, _D),
        "jdeposition": fn("jdeposition", None, C.c_void_p, _DP, _DP, _D),
        "zero_j": fn("zero_j", None, C.c_void_p),
        "gather": fn("gather", None, C.c_void_p, _D, _D, _D, _DP, _DP),
        "chi": fn("chi", _D, C.c_void_p, _DP, _DP, _DP, _D),
        "w": fn("w", _D, C.c_void_p, _D, _DP, _D),
        "tilde_w": fn("tilde_w", _D, C.c_void_p, _D, _D, _D),
        "mathcal_W": fn("mathcal_W", _D, C.c_void_p, _DP, _DP),
        "get_rand": fn("get_rand", _D, C.c_void_p),
        "pmerging": fn("pmerging", None, C.c_void_p, C.c_int, _DP),
        "moving_window": fn("moving_window", None, C.c_void_p),
        "set_diag_range": fn("set_diag_range", None, C.c_void_p, C.c_int, C.c_int),
        "get_field_slab": fn("get_field_slab", None, C.c_void_p, C.c_int, C.c_int, _DP),
        "set_field_slab": fn("set_field_slab", None, C.c_void_p, C.c_int, C.c_int, _DP),
        "get_particle_slab": fn("get_particle_slab", C.c_long, C.c_void_p, C.c_int, C.c_int, C.c_long, _DP, _LP),
        "replace_particle_slab": fn("replace_particle_slab", None, C.c_void_p, C.c_int, C.c_int, C.c_long,
                                    _DP, _DP, _DP, _DP, _DP, _DP, _DP, _DP, _DP, _DP),
        "layer_counts": fn("layer_counts", None, C.c_void_p, _LP),
    }
    if kind == "ref":
        _IP = C.POINTER(C.c_int)
        api["optimal_partition"] = fn("optimal_partition", None, _DP, C.c_int, C.c_int, C.c_int, _IP)
        api["normalize_partition"] = fn("normalize_partition", None, _IP, _IP, C.c_int, C.c_int, _IP)
        api["partition_imbalance"] = fn("partition_imbalance", _D, _DP, C.c_int, _IP, C.c_int, C.c_int)
        I = C.c_int
        api["f_init_cos"] = fn("f_init_cos", None, C.c_void_p, _D, _D, _D, _D, _D, _D, I, I, _D, _D, _D, _D, I, _D,
                               _D, _D, _D)
        api["f_init_focused"] = fn("f_init_focused", None, C.c_void_p, _D, _D, _D, _D, _D, _D, I, _D, _D, _D, I, _D,
                                   I, _D, _D, _D, _D)
        api["set_catching"] = fn("set_catching", None, C.c_void_p, I)
        api["energy_deleted"] = fn("energy_deleted", None, C.c_void_p, _DP)
    _LIBS[key] = api
    return api


def _dp(a: np.ndarray):
    return a.ctypes.data_as(_DP)


PARTICLE_KEYS = ("x", "y", "z", "ux", "uy", "uz", "g", "q", "cmr", "chi")
FIELD_KEYS = ("ex", "ey", "ez", "bx", "by", "bz", "jx", "jy", "jz", "bex", "bey", "bez")


class Region:
    """One simulation region on the CPU checker (reference or restatement)."""

    def __init__(self, nx, ny, nz, dx, dy, dz, dt, *, lambda_cm=1e-4, solver=0, pusher=1,
                 qed=False, icmr=(), seed=0, kind="port", flavour="parity"):
        self.api = _load(kind, flavour)
        self.kind = kind
        self.shape = (nx, ny, nz)
        self.dx, self.dy, self.dz, self.dt = dx, dy, dz, dt
        ic = np.ascontiguousarray(np.asarray(icmr, dtype=np.float64).reshape(-1))
        if ic.size == 0:
            ic = np.zeros(1)
            n_ion = 0
        else:
            n_ion = ic.size
        self._icmr = ic
        self.n_ion = n_ion
        self.h = self.api["create"](nx, ny, nz, dx, dy, dz, dt, lambda_cm, solver, pusher,
                                    int(bool(qed)), n_ion, _dp(ic), int(seed))

    def close(self):
        if self.h:
            self.api["destroy"](self.h)
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
        self.api["set_fields"](self.h, *[_dp(a) for a in arrs])

    def get_fields(self) -> np.ndarray:
        out = np.empty((12,) + self.shape, dtype=np.float64)
        self.api["get_fields"](self.h, _dp(out))
        return out

    def init_boundaries(self):
        self.api["init_boundaries"](self.h)

    def add_particles(self, parts: dict):
        n = len(parts["x"])
        arrs = []
        for k in PARTICLE_KEYS:
            a = parts.get(k)
            if a is None:
                a = np.zeros(n)
            arrs.append(np.ascontiguousarray(a, dtype=np.float64))
        self.api["add_particles"](self.h, n, *[_dp(a) for a in arrs])

    def count(self) -> int:
        return self.api["count_particles"](self.h)

    def get_particles(self):
        n = self.count()
        cap = max(n, 1)
        out = np.empty((10, cap), dtype=np.float64)
        cell = np.empty(cap, dtype=np.int64)
        self.api["get_particles"](self.h, cap, _dp(out), cell.ctypes.data_as(_LP))
        d = {k: out[i, :n].copy() for i, k in enumerate(PARTICLE_KEYS)}
        d["cell"] = cell[:n].copy()
        return d

    def diag_len(self) -> int:
        return self.api["diag_len"](self.h)

    def step(self, nsteps=1, external_bz=0.0) -> np.ndarray:
        d = np.zeros((nsteps, self.diag_len()), dtype=np.float64)
        self.api["step"](self.h, nsteps, external_bz, _dp(d))
        return d

    def padvance(self, external_bz=0.0):
        self.api["padvance"](self.h, external_bz)

    def fadvance(self):
        self.api["fadvance"](self.h)

    def compute_diag(self) -> np.ndarray:
        d = np.zeros(self.diag_len())
        self.api["compute_diag"](self.h, _dp(d))
        return d

    def zero_j(self):
        self.api["zero_j"](self.h)

    def jdeposition(self, pos, d, q):
        p = np.ascontiguousarray(pos, dtype=np.float64).copy()
        dd = np.ascontiguousarray(d, dtype=np.float64)
        self.api["jdeposition"](self.h, _dp(p), _dp(dd), q)
        return p

    def gather(self, x, y, z):
        e = np.zeros(3)
        b = np.zeros(3)
        self.api["gather"](self.h, x, y, z, _dp(e), _dp(b))
        return e, b

    def chi(self, e, b, u, g):
        e, b, u = (np.ascontiguousarray(v, dtype=np.float64) for v in (e, b, u))
        return self.api["chi"](self.h, _dp(e), _dp(b), _dp(u), g)

    def w(self, g, r, chi):
        rr = np.array([r], dtype=np.float64)
        v = self.api["w"](self.h, g, _dp(rr), chi)
        return v, float(rr[0])

    def tilde_w(self, g, r, chi):
        return self.api["tilde_w"](self.h, g, r, chi)

    def mathcal_W(self, e, b):
        e, b = (np.ascontiguousarray(v, dtype=np.float64) for v in (e, b))
        return self.api["mathcal_W"](self.h, _dp(e), _dp(b))

    def get_rand(self):
        return self.api["get_rand"](self.h)

    def moving_window(self):
        """spatial_region::moving_window: shift everything one cell towards -x."""
        self.api["moving_window"](self.h)

    def pmerging(self, mode: str, ppd):
        """spatial_region::pmerging; mode "ti" or "nl", ppd per class
        (electrons, positrons, photons, then the ion populations)."""
        p = np.zeros(3 + self.n_ion)
        v = np.asarray(ppd, dtype=np.float64).reshape(-1)
        p[:min(v.size, p.size)] = v[:p.size]
        self.api["pmerging"](self.h, 1 if mode == "ti" else 2, _dp(p))


    # --- x-slabs (the n_sr > 1 exchange, main.cpp:1286-1514) ---------------
    # The CPU checkers keep all species in one list per cell, so a slab is
    # exchanged for all species at once (species=None).
    species_ids = (None,)

    def set_diag_range(self, i_lo: int, i_hi: int):
        self.api["set_diag_range"](self.h, int(i_lo), int(i_hi))

    def get_field_slab(self, i0: int, width: int) -> np.ndarray:
        out = np.zeros((12, width) + self.shape[1:])
        self.api["get_field_slab"](self.h, i0, width, _dp(out))
        return out

    def set_field_slab(self, i0: int, planes12: np.ndarray):
        a = np.ascontiguousarray(planes12, dtype=np.float64)
        self.api["set_field_slab"](self.h, i0, a.size // (12 * self.shape[1] * self.shape[2]), _dp(a))

    def get_particle_slab(self, species, i0: int, width: int) -> dict:
        n = self.api["get_particle_slab"](self.h, i0, width, 0, None, None)
        cap = max(n, 1)
        out = np.zeros((10, cap))
        self.api["get_particle_slab"](self.h, i0, width, cap, _dp(out), None)
        return {k: out[i, :n].copy() for i, k in enumerate(PARTICLE_KEYS)}

    def replace_particle_slab(self, species, i0: int, width: int, parts: dict):
        n = len(parts["x"])
        arrs = [np.ascontiguousarray(parts[k] if parts.get(k) is not None else np.zeros(n), dtype=np.float64)
                for k in PARTICLE_KEYS]
        self.api["replace_particle_slab"](self.h, i0, width, n, *[_dp(a) for a in arrs])

    # --- initial pulses (reference only; the reference's argument order) ---
    def f_init_cos(self, a0y, a0z, xsigma, ysigma, zsigma, x0, sscos, b_sign, x1, phase, y0, z0, append, phi,
                   xtarget=0.0, ytarget=0.0, ztarget=0.0):
        """f_init_cos (init.cpp:6-210)."""
        self.api["f_init_cos"](self.h, a0y, a0z, xsigma, ysigma, zsigma, x0, int(sscos), int(b_sign), x1, phase,
                               y0, z0, int(append), phi, xtarget, ytarget, ztarget)

    def f_init_focused(self, a0y, a0z, xsigma, sigma0, x0, x1, b_sign, phase, y0, z0, append, phi, sscos, K,
                       xtarget=0.0, ytarget=0.0, ztarget=0.0):
        """f_init_focused (init.cpp:212-385)."""
        self.api["f_init_focused"](self.h, a0y, a0z, xsigma, sigma0, x0, x1, int(b_sign), phase, y0, z0,
                                   int(append), phi, int(sscos), K, xtarget, ytarget, ztarget)

    # --- catching (reference only) ----------------------------------------
    def set_catching(self, on: bool):
        """catching_enabled: erased particles' energy is summed by the
        reference's update_energy_deleted (a process-wide flag)."""
        self.api["set_catching"](self.h, int(bool(on)))

    def energy_deleted(self) -> np.ndarray:
        """Cumulative deleted energies in Joules: electrons, positrons,
        photons, then each ion population."""
        out = np.zeros(3 + self.n_ion)
        self.api["energy_deleted"](self.h, _dp(out))
        return out

    def layer_counts(self) -> np.ndarray:
        out = np.zeros(self.shape[0], dtype=np.int64)
        self.api["layer_counts"](self.h, out.ctypes.data_as(_LP))
        return out


def ref_optimal_partition(weights, regions: int, overlap: int) -> list:
    """The reference's calculate_optimal_partition (balancing.cpp:54-115)."""
    api = _load("ref", "parity")
    w = np.ascontiguousarray(weights, dtype=np.float64)
    out = (C.c_int * regions)()
    api["optimal_partition"](_dp(w), w.size, regions, overlap, out)
    return list(out)


def ref_normalize_partition(old, new, overlap: int) -> list:
    """The reference's normalize_new_partition (balancing.cpp:136-175)."""
    api = _load("ref", "parity")
    n = len(old)
    a, b, out = (C.c_int * n)(*old), (C.c_int * n)(*new), (C.c_int * n)()
    api["normalize_partition"](a, b, n, overlap, out)
    return list(out)


def ref_partition_imbalance(weights, partition, overlap: int) -> float:
    """The reference's calculate_partition_imbalance (balancing.cpp:132-134)."""
    api = _load("ref", "parity")
    w = np.ascontiguousarray(weights, dtype=np.float64)
    p = (C.c_int * len(partition))(*partition)
    return api["partition_imbalance"](_dp(w), w.size, p, len(partition), overlap)


def push(pusher, cmr, state, e, b, dt, kind="port", flavour="parity"):
    api = _load(kind, flavour)
    s = np.ascontiguousarray(state, dtype=np.float64).copy()
    e, b = (np.ascontiguousarray(v, dtype=np.float64) for v in (e, b))
    api["push"](pusher, cmr, _dp(s), _dp(e), _dp(b), dt)
    return s
