"""GPU test of kg_relatedness_noalloc, the entry point for callers that cannot
allocate device memory.  Collected last (file name) so a run that stops at the
first failure has already run every other test.

The caller owns both device buffers (allocated here with torch, standing in
for the caller's own pool); the entry point must produce the rows of the
allocating entry point kg_relatedness on the same cohort, within the tolerances
the other parity tests use, on two calls in a row (the shared scratch array
keeps the previous call's contents)."""
import ctypes

import numpy as np
import pytest

import kestrel_b200 as kb
from kestrel_b200 import _lib, synth

pytestmark = pytest.mark.gpu


def _noalloc_rows(codes, iterations=100):
    import torch
    n, m = codes.shape
    np_ = n * (n + 1) // 2
    d_codes = torch.from_numpy(codes).to("cuda:0")
    d_out = torch.zeros(np_ * kb.OUTPUT_DTYPE.itemsize, dtype=torch.uint8, device="cuda:0")
    stream = torch.cuda.current_stream().cuda_stream
    st = _lib.lib().kg_relatedness_noalloc(ctypes.c_void_p(d_codes.data_ptr()), n, m, m, iterations,
                                           float("nan"), ctypes.c_void_p(d_out.data_ptr()), np_,
                                           ctypes.c_void_p(stream))
    assert st == 0, _lib.STATUS_NAMES.get(st, st)
    torch.cuda.synchronize()
    return d_out.cpu().numpy().view(kb.OUTPUT_DTYPE)


def _check_close(a, b):
    assert np.array_equal(a["x"], b["x"]) and np.array_equal(a["y"], b["y"])
    assert np.abs(a["jacquard"] - b["jacquard"]).max() <= 1e-5
    assert (np.abs(a["obj"] - b["obj"]) / np.abs(b["obj"])).max() <= 1e-6
    la, lb = np.log10(a["cond"]), np.log10(b["cond"])
    below = np.isfinite(lb) & (lb < 15)
    assert np.all((la[below] > 15) == (lb[below] > 15))


def test_noalloc_matches_allocating_entry_point():
    cohorts = [synth.make_cohort(40, 6000, seed=31, planted={"parent_offspring": 2, "full_sib": 2}),
               synth.make_cohort(24, 3000, seed=32, missing=0.05)]
    with kb.Estimator() as est:
        for c in cohorts:                      # two calls in a row, different shapes
            est.load(c.codes)
            ref = est.relatedness()
            got = _noalloc_rows(c.codes)
            _check_close(got, ref)
        got2 = _noalloc_rows(cohorts[1].codes)  # and the same call again
        _check_close(got2, ref)


def test_noalloc_matches_the_oracle(oracle):
    """The same rows against the FP64 oracle directly (the bar of the other
    parity tests)."""
    from .parity import compare
    c = synth.make_cohort(32, 5000, seed=33, planted={"half_sib": 2})
    print(compare(_noalloc_rows(c.codes), oracle.relatedness(c.codes)))


def test_noalloc_rejects_oversized_input():
    import torch
    codes = torch.zeros((513, 10), dtype=torch.uint8, device="cuda:0")
    out = torch.zeros(16, dtype=torch.uint8, device="cuda:0")
    st = _lib.lib().kg_relatedness_noalloc(ctypes.c_void_p(codes.data_ptr()), 513, 10, 10, 100,
                                           float("nan"), ctypes.c_void_p(out.data_ptr()), 1, None)
    assert st in (_lib.KG_ENOMEM, _lib.KG_EINVAL)
    st = _lib.lib().kg_relatedness_noalloc(ctypes.c_void_p(codes.data_ptr()), 4, 40000, 40000, 100,
                                           float("nan"), ctypes.c_void_p(out.data_ptr()), 10, None)
    assert st == _lib.KG_ENOMEM
