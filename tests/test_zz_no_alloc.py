"""qp_eval_qed_rates_noalloc, the entry point for callers that cannot
allocate GPU memory (their device memory belongs to another allocator), must
give the same results as qp_eval_qed_rates, which stages its data in buffers
it allocates on every call.  Two calls in a row with different inputs check
that the shared staging array carries nothing over from one call to the
next.  This file sorts last so that a failure here comes after every other
test has run."""
import ctypes as C

import numpy as np
import pytest

from tests.conftest import gpu_available

MAX_SAMPLES = 16384


def _samples(n, seed):
    rng = np.random.default_rng(seed)
    e = rng.standard_normal((n, 3)) * 10 ** rng.uniform(1, 5, (n, 1))
    b = rng.standard_normal((n, 3)) * 10 ** rng.uniform(1, 5, (n, 1))
    u = rng.standard_normal((n, 3)) * 10 ** rng.uniform(0, 3.5, (n, 1))
    g = np.sqrt(1 + (u * u).sum(1))
    r = rng.uniform(0, 1, n)
    chi = 10 ** rng.uniform(-3, 1, n)
    return np.ascontiguousarray(np.column_stack([e, b, u, g, r, chi]))


def _call(lib, name, smp):
    out = np.full((smp.shape[0], 5), np.nan)
    dp = C.POINTER(C.c_double)
    r = getattr(lib, name)(0, 1e-4, smp.shape[0], smp.ctypes.data_as(dp), out.ctypes.data_as(dp))
    assert r == 0, lib.qp_last_error(None)
    return out


@pytest.mark.gpu
def test_noalloc_rates_match_allocating_entry_point():
    if not gpu_available():
        pytest.skip("no CUDA device")
    from quill_b200.api import load_library
    lib = load_library()
    for call, (n, seed) in enumerate([(5000, 21), (MAX_SAMPLES, 22)]):
        smp = _samples(n, seed)
        ref = _call(lib, "qp_eval_qed_rates", smp)
        got = _call(lib, "qp_eval_qed_rates_noalloc", smp)
        # same kernel on the same inputs: equal to the tolerance of the
        # other rate tests (1e-11 relative)
        np.testing.assert_allclose(got, ref, rtol=1e-11, atol=1e-300, err_msg=f"call {call}")
        assert not np.isnan(got).any()


@pytest.mark.gpu
def test_noalloc_rejects_oversize_request():
    if not gpu_available():
        pytest.skip("no CUDA device")
    from quill_b200.api import load_library
    lib = load_library()
    smp = _samples(4, 23)
    out = np.zeros((4, 5))
    dp = C.POINTER(C.c_double)
    r = lib.qp_eval_qed_rates_noalloc(0, 1e-4, MAX_SAMPLES + 1, smp.ctypes.data_as(dp), out.ctypes.data_as(dp))
    assert r == 7  # QP_ERR_ARG
    assert b"exceed" in lib.qp_last_error(None)
