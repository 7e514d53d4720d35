"""The device random numbers: philox4x32_10 (quill_b200/csrc/qp_qed.cuh)
against the three known-answer vectors published with Random123 for
Philox4x32 with 10 rounds.  The function is __host__ __device__; the test
compiles it as host code (no GPU needed)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# (counter, key) -> output, Random123 kat_vectors "philox4x32 10"
KAT = [
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]

PROG = r"""
#include <cstdio>
#include "qp_qed.cuh"
int main(int argc, char** argv) {
    unsigned v[6];
    for (int i = 0; i < 6; i++) sscanf(argv[1 + i], "%x", &v[i]);
    qp::Philox4 p = qp::philox4x32_10(v[0], v[1], v[2], v[3], v[4], v[5]);
    printf("%08x %08x %08x %08x\n", p.v[0], p.v[1], p.v[2], p.v[3]);
    return 0;
}
"""


def test_philox_known_answers(tmp_path):
    cxx = shutil.which("g++")
    cuda_inc = "/usr/local/cuda/include"
    if cxx is None or not os.path.isdir(cuda_inc):
        pytest.skip("needs g++ and the CUDA headers")
    src = tmp_path / "kat.cpp"
    src.write_text(PROG)
    exe = tmp_path / "kat"
    subprocess.run([cxx, "-O2", "-std=c++17", f"-I{cuda_inc}", f"-I{os.path.join(ROOT, 'quill_b200', 'csrc')}",
                    f"-I{os.path.join(ROOT, 'include')}", str(src), "-o", str(exe)], check=True)
    for ctr, key, want in KAT:
        args = [f"{x:08x}" for x in ctr + key]
        out = subprocess.run([str(exe)] + args, check=True, capture_output=True, text=True).stdout.split()
        assert tuple(int(w, 16) for w in out) == want
