"""Error paths of the bounded wave loops, exercised without a GPU fault.

A call's waves are bounded (kg_set_wave_limit; by default a bound from the
work that only stops a loop that would not end).  Here the bound is set to two
waves on a cohort that needs many more: the call must return KG_ETIMEOUT with
the device and the context still usable, and the next call on the same
context must give the oracle's rows, bit for bit those of a fresh context.
Both wave drivers are covered: the device loop (one graph launch per call)
and host-driven waves (KESTREL_HOST_WAVES=1)."""
import os

import numpy as np
import pytest

import kestrel_b200 as kb
from kestrel_b200 import synth

from .parity import compare

pytestmark = pytest.mark.gpu


def _bitwise_equal(a, b):
    return a.shape == b.shape and np.array_equal(a.view(np.uint8), b.view(np.uint8))


@pytest.mark.parametrize("host_waves", [False, True])
def test_wave_limit_times_out_and_the_context_recovers(oracle, host_waves, monkeypatch):
    if host_waves:
        monkeypatch.setenv("KESTREL_HOST_WAVES", "1")
    else:
        monkeypatch.delenv("KESTREL_HOST_WAVES", raising=False)
    co = synth.make_cohort(48, 4000, seed=61, planted={"full_sib": 2})
    with kb.Estimator() as fresh:
        fresh.load(co.codes)
        want = fresh.relatedness()
    with kb.Estimator() as est:
        est.load(co.codes)
        est.set_wave_limit(2)
        with pytest.raises(kb.KestrelError) as ei:
            est.relatedness()
        assert ei.value.status == kb.KG_ETIMEOUT
        assert "wave limit" in str(ei.value)
        est.set_wave_limit(0)
        got = est.relatedness()
        assert est.run_stats()["waves"] > 2
    assert _bitwise_equal(got, want)
    print(compare(got, oracle.relatedness(co.codes)))
    assert os.environ.get("KESTREL_HOST_WAVES") == ("1" if host_waves else None)
