"""Reference output files of the driver's end-to-end test (test infrastructure).

For every conf under tests/golden/driver/ this runs, here where the
reference's sources are present:

    python3 <reference>/parse.py <conf>            -> <name>.stream  (committed)
    oracle/_ref/quill < <name>.stream              -> its output files

and stores every output file except `log` (which holds wall-clock times)
byte for byte in <name>_ref.npz (one uint8 array per file name).
oracle/_ref/quill is the reference's own complete program built by
`make -C oracle quill` (one process, n_sr = 1).  The test replays the
committed stream through qp_driver on the GPU and compares the files.

    python tests/golden/make_driver_golden.py
"""
import glob
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF_ROOT = os.environ.get("QUILL_REF_ROOT", "/root/reference")


def main():
    quill = os.path.join(ROOT, "oracle", "_ref", "quill")
    if not os.path.exists(quill):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "quill", f"REF_ROOT={REF_ROOT}"], check=True)
    for conf in sorted(glob.glob(os.path.join(HERE, "driver", "*.conf"))):
        name = os.path.splitext(os.path.basename(conf))[0]
        stream = subprocess.run([sys.executable, os.path.join(REF_ROOT, "parse.py"), conf], check=True,
                                capture_output=True, text=True).stdout
        with open(os.path.join(HERE, "driver", name + ".stream"), "w") as f:
            f.write(stream)
        with tempfile.TemporaryDirectory() as d:
            os.makedirs(os.path.join(d, "results"))
            subprocess.run([quill], input=stream, text=True, cwd=d, check=True, capture_output=True)
            files = {}
            for p in sorted(os.listdir(os.path.join(d, "results"))):
                if p == "log":
                    continue
                with open(os.path.join(d, "results", p), "rb") as f:
                    files[p] = np.frombuffer(f.read(), dtype=np.uint8)
        np.savez_compressed(os.path.join(HERE, "driver", name + "_ref.npz"), **files)
        print(f"{name}: {len(files)} files")


if __name__ == "__main__":
    main()
