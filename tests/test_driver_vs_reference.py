"""The driver end to end against the reference's own program.

tests/golden/driver/<name>.stream is the record stream the reference's
parse.py made of <name>.conf; <name>_ref.npz holds every output file the
reference's complete program (its src/main.cpp, one process) wrote for it
(tests/golden/make_driver_golden.py).  Here qp_driver reads the same stream
on the GPU and every file the reference wrote must exist with the same
number of values, equal to the 6 significant digits of the text output: a
value is equal if its text is identical, or if it differs from the
reference's by no more than the rounding of 6 digits (5e-6 relative, for a
last digit that rounds the other way) or by 1e-9 of the file's largest
magnitude (values that are round-off next to the file's scale, such as a
field component that is zero in the reference and 1e-17 here).

* laser: a pulse in vacuum, FDTD + Boris: field files, w, inv, currents
  and the empty densities, spectra and phase-space files.
* film: the pulse on a cold electron film with the driver's reference-order
  current (current_order = reference): densities, currents, spectra and
  every written phase-space particle as well.
"""
import os
import subprocess

import numpy as np
import pytest

from tests.conftest import gpu_available

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden", "driver")
DRIVER = os.path.join(os.path.dirname(HERE), "quill_b200", "qp_driver")


def _values(text: bytes):
    return [ln for ln in text.decode().split("\n") if ln != ""]


def compare_file(name, ours: bytes, ref: bytes):
    a, b = _values(ours), _values(ref)
    assert len(a) == len(b), f"{name}: {len(a)} values, the reference wrote {len(b)}"
    if a == b:
        return 0
    fa = np.array([float(x) for x in a])
    fb = np.array([float(x) for x in b])
    scale = float(np.max(np.abs(fb))) if fb.size else 0.0
    diff = np.abs(fa - fb)
    ok = (diff <= 5e-6 * np.maximum(np.abs(fa), np.abs(fb))) | (diff <= 1e-9 * scale)
    bad = np.flatnonzero(~ok)
    assert bad.size == 0, (f"{name}: {bad.size} of {fa.size} values differ, first at {bad[0]}: "
                           f"{a[bad[0]]} vs reference {b[bad[0]]}")
    return int(np.count_nonzero(np.array(a) != np.array(b)))


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["laser", "film"])
def test_driver_files_equal_reference(name, tmp_path):
    if not gpu_available():
        pytest.skip("no CUDA device")
    with open(os.path.join(GOLD, name + ".stream")) as f:
        stream = f.read()
    os.makedirs(tmp_path / "results")
    r = subprocess.run([DRIVER], input=stream, text=True, cwd=tmp_path, capture_output=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    ref = np.load(os.path.join(GOLD, name + "_ref.npz"))
    ours = set(os.listdir(tmp_path / "results"))
    missing = sorted(set(ref.files) - ours)
    assert not missing, f"files the reference writes and the driver does not: {missing}"
    not_bitwise = {}
    for fname in ref.files:
        with open(tmp_path / "results" / fname, "rb") as f:
            n = compare_file(fname, f.read(), ref[fname].tobytes())
        if n:
            not_bitwise[fname] = n
    print(f"{name}: {len(ref.files)} files equal to 6 digits; values whose text differs in the last digit: "
          f"{not_bitwise}")
