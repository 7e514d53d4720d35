"""qp_eval_qed_rates_noalloc, the entry point for callers that cannot
allocate GPU memory (their device memory belongs to another allocator), must
give the same results as qp_eval_qed_rates, which stages its data in buffers
it allocates on every call.  Calls in a row with different inputs (a
smaller one after the largest) check that the shared staging array carries
nothing over from one call to the next; the rows past n of the output must
stay untouched.  Around the calls the device's free memory must not change,
and a call must still succeed when the device has almost no free memory
left.  This file sorts last so that a failure here comes after every other
test has run."""
import ctypes as C

import numpy as np
import pytest

from tests.conftest import gpu_available

MAX_SAMPLES = 16384
dp = C.POINTER(C.c_double)


def _samples(n, seed):
    rng = np.random.default_rng(seed)
    e = rng.standard_normal((n, 3)) * 10 ** rng.uniform(1, 5, (n, 1))
    b = rng.standard_normal((n, 3)) * 10 ** rng.uniform(1, 5, (n, 1))
    u = rng.standard_normal((n, 3)) * 10 ** rng.uniform(0, 3.5, (n, 1))
    g = np.sqrt(1 + (u * u).sum(1))
    r = rng.uniform(0, 1, n)
    chi = 10 ** rng.uniform(-3, 1, n)
    return np.ascontiguousarray(np.column_stack([e, b, u, g, r, chi]))


def _call(lib, name, smp, spare_rows=0):
    n = smp.shape[0]
    out = np.full((n + spare_rows, 5), np.nan)
    r = getattr(lib, name)(0, 1e-4, n, smp.ctypes.data_as(dp), out.ctypes.data_as(dp))
    assert r == 0, lib.qp_last_error(None)
    assert np.isnan(out[n:]).all(), f"{name} wrote past the {n} requested rows"
    return out[:n]


def _lib():
    if not gpu_available():
        pytest.skip("no CUDA device")
    from quill_b200.api import load_library
    return load_library()


@pytest.mark.gpu
def test_noalloc_rates_match_allocating_entry_point():
    import torch
    lib = _lib()
    torch.cuda.init()
    # one call first: the library's device code (and with it the staging
    # array) is loaded on first use
    _call(lib, "qp_eval_qed_rates_noalloc", _samples(8, 20))
    torch.cuda.synchronize()
    for call, (n, seed) in enumerate([(5000, 21), (MAX_SAMPLES, 22), (777, 24)]):
        smp = _samples(n, seed)
        ref = _call(lib, "qp_eval_qed_rates", smp, spare_rows=3)
        got = _call(lib, "qp_eval_qed_rates_noalloc", smp, spare_rows=3)
        # same kernel on the same inputs: equal to the tolerance of the
        # other rate tests (1e-11 relative)
        np.testing.assert_allclose(got, ref, rtol=1e-11, atol=1e-300, err_msg=f"call {call}")
        assert not np.isnan(got).any()
        before = torch.cuda.mem_get_info(0)[0]
        _call(lib, "qp_eval_qed_rates_noalloc", smp)
        assert torch.cuda.mem_get_info(0)[0] == before, f"call {call}: free device memory changed"


@pytest.mark.gpu
def test_noalloc_runs_on_a_full_device():
    """With the device's free memory held by another allocator (torch here)
    down to less than the allocating entry point would need for the call,
    the entry point that allocates nothing still runs and gives the same
    results."""
    import torch
    lib = _lib()
    smp = _samples(MAX_SAMPLES, 25)
    ref = _call(lib, "qp_eval_qed_rates", smp)
    _call(lib, "qp_eval_qed_rates_noalloc", smp)  # loaded before the device fills
    need = smp.nbytes + MAX_SAMPLES * 5 * 8
    held = []
    try:
        chunk = 1 << 30
        while chunk >= (1 << 12):  # small tensors take 2 MB segments: the last ones fill the gaps
            try:
                held.append(torch.empty(chunk, dtype=torch.uint8, device="cuda:0"))
            except torch.OutOfMemoryError:
                chunk >>= 1
        free = torch.cuda.mem_get_info(0)[0]
        if free >= need:
            pytest.skip(f"could not fill the device ({free} bytes still free)")
        got = _call(lib, "qp_eval_qed_rates_noalloc", smp)
        np.testing.assert_allclose(got, ref, rtol=1e-11, atol=1e-300)
    finally:
        held.clear()
        torch.cuda.empty_cache()


@pytest.mark.gpu
def test_noalloc_rejects_oversize_request():
    lib = _lib()
    smp = _samples(4, 23)
    out = np.zeros((4, 5))
    r = lib.qp_eval_qed_rates_noalloc(0, 1e-4, MAX_SAMPLES + 1, smp.ctypes.data_as(dp), out.ctypes.data_as(dp))
    assert r == 7  # QP_ERR_ARG
    assert b"exceed" in lib.qp_last_error(None)
