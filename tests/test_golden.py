"""The committed golden vectors (tests/golden/*.npz, made from the
reference's own sources by tests/golden/make_golden.py) pin the C
restatement bit for bit and the CUDA FP64 path to 1e-12 (bit-exact cell
order), without needing the reference sources at run time."""
import glob
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.conftest import gpu_available

HERE = os.path.dirname(os.path.abspath(__file__))
FILES = sorted(glob.glob(os.path.join(HERE, "golden", "golden_*.npz")))
FK = ("ex", "ey", "ez", "bx", "by", "bz")
STEPS = 3


def _load(path):
    return dict(np.load(path))


@pytest.mark.parametrize("path", FILES, ids=[os.path.basename(f) for f in FILES])
def test_port_matches_golden(path):
    if not O.available("port", "parity"):
        import subprocess
        subprocess.run(["make", "-C", os.path.join(os.path.dirname(HERE), "oracle")], check=True,
                       capture_output=True)
    g = _load(path)
    nx, ny, nz = (int(v) for v in g["grid"])
    reg = O.Region(nx, ny, nz, float(g["dx"]), float(g["dx"]), float(g["dx"]), float(g["dt"]),
                   solver=int(g["solver"]), pusher=int(g["pusher"]), icmr=(1 / 1836.15,), seed=7, kind="port")
    reg.set_fields(*[g["in_" + k] for k in FK])
    reg.init_boundaries()
    reg.add_particles({k: g["in_p_" + k] for k in O.PARTICLE_KEYS})
    for s in range(STEPS):
        d = reg.step(1, external_bz=float(g["external_bz"]))[0]
        np.testing.assert_array_equal(reg.get_fields(), g[f"s{s}_fields"])
        p = reg.get_particles()
        for k in O.PARTICLE_KEYS:
            np.testing.assert_array_equal(p[k], g[f"s{s}_p_{k}"])
        np.testing.assert_array_equal(p["cell"], g[f"s{s}_p_cell"])
        np.testing.assert_array_equal(d, g[f"s{s}_diag"])


@pytest.mark.gpu
@pytest.mark.parametrize("path", FILES, ids=[os.path.basename(f) for f in FILES])
def test_cuda_matches_golden(path):
    if not gpu_available():
        pytest.skip("no CUDA device")
    from quill_b200.api import Region
    g = _load(path)
    nx, ny, nz = (int(v) for v in g["grid"])
    species = (-1.0, 1.0, 1 / 1836.15, 0.0)
    reg = Region(nx, ny, nz, float(g["dx"]), float(g["dx"]), float(g["dx"]), float(g["dt"]), species_cmr=species,
                 solver=int(g["solver"]), pusher=int(g["pusher"]))
    reg.set_fields(*[g["in_" + k] for k in FK])
    reg.init_boundaries()
    cmr_in = g["in_p_cmr"]
    for si, c in enumerate(species):
        sel = cmr_in == c
        reg.add_particles(si, {k: g["in_p_" + k][sel] for k in ("x", "y", "z", "ux", "uy", "uz", "g", "q")})
    for s in range(STEPS):
        d = reg.step(1, external_bz=float(g["external_bz"]))[0]
        f = reg.get_fields()
        ref = g[f"s{s}_fields"]
        for a in range(12):
            scale = np.max(np.abs(ref[a])) or 1.0
            assert np.max(np.abs(f[a] - ref[a])) / scale <= 1e-12, (s, a)
        cm = g[f"s{s}_p_cmr"]
        for si, c in enumerate(species):
            p = reg.get_particles(si)
            sel = cm == c
            np.testing.assert_array_equal(p["cell"], g[f"s{s}_p_cell"][sel])
            for k in ("x", "y", "z", "ux", "uy", "uz", "g"):
                ref_k = g[f"s{s}_p_{k}"][sel]
                if s == 0:
                    np.testing.assert_array_equal(p[k], ref_k)
                else:
                    scale = np.max(np.abs(ref_k)) if ref_k.size else 1.0
                    assert np.max(np.abs(p[k] - ref_k), initial=0.0) <= 1e-12 * scale
        np.testing.assert_allclose(d.as_array(), g[f"s{s}_diag"], rtol=1e-12)
