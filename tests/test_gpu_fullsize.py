"""GPU parity at the full sizes of the uneven-cohort batch and the inbred stress
cohort, through the C ABI, against the FP64 oracle (the bar of tests/parity.py:
Delta and kinship within 1e-5 and the objective within 1e-6 relative wherever
the oracle's log10 condition estimate is below 15, the condition flag equal
there).

* Inbred / ill-conditioned stress, N=512 x M=50,000 (128 inbred samples, 32
  identical-inbred pairs, a 5,000-site low-information block): every one of
  the 131,328 rows (130,816 pairs + 512 self pairs) against the oracle, so the
  pairs the GPU re-evaluated in FP64 and any pair with an oracle log10 cond
  between 4 and 15 are all in the comparison.
* Eight uneven cohorts in one launch (N = 96 .. 2048, M = 20k .. 100k,
  per-sample missingness U(0, 0.2); 3,168,704 pairs): 100 random pairs and 4
  self pairs of every cohort against the oracle with that cohort's own
  frequencies, and the size-independent properties of every row."""
import numpy as np
import pytest

import kestrel_b200 as kb
from kestrel_b200 import synth

from .parity import compare

pytestmark = pytest.mark.gpu


def _simplex_rows_ok(rows):
    jac = rows["jacquard"]
    assert np.all(jac >= 0.0) and np.abs(jac.sum(1) - 1.0).max() < 1e-12
    assert np.all(np.isfinite(rows["obj"]))
    kin = jac @ kb.KINSHIP_VECTOR
    assert kin.min() >= 0.0 and kin.max() <= 1.0 + 1e-12


def test_inbred_stress_full_size_every_pair(oracle):
    co = synth.config3()
    n = co.codes.shape[0]
    with kb.Estimator() as est:
        est.load(co.codes)
        gpu = est.relatedness()
        st = est.run_stats()
    assert len(gpu) == n * (n + 1) // 2
    _simplex_rows_ok(gpu)
    ref = oracle.relatedness(co.codes)
    out = compare(gpu, ref)
    lc = np.log10(ref["cond"])
    print(out, {"fp64_pairs": st["fp64_pairs"], "oracle_flagged": int(np.sum(~(lc < 15)))})
    assert st["fp64_pairs"] > 0, "the stress cohort should send pairs to FP64 passes"
    assert np.any(~(lc < 15)), "the stress cohort should hold flagged pairs"
    pos = {(int(a), int(b)): i for i, (a, b) in enumerate(zip(gpu["x"], gpu["y"]))}
    for a, b, rel, _ in co.planted:
        assert gpu["jacquard"][pos[(a, b)]][0] > 0.9, (a, b, rel)


def test_uneven_cohorts_full_size(oracle):
    cohorts = synth.config2()
    with kb.Estimator() as est:
        outs = est.relatedness_batch([(c.codes,) for c in cohorts])
        st = est.run_stats()
    rng = np.random.default_rng(17)
    summary = []
    for c, rows in zip(cohorts, outs):
        n = c.codes.shape[0]
        assert len(rows) == n * (n + 1) // 2
        _simplex_rows_ok(rows)
        idx = rng.choice(len(rows), 100, replace=False)
        xs, ys = rows["x"].astype(np.int64), rows["y"].astype(np.int64)
        self_idx = np.nonzero(xs == ys)[0][:4]
        idx = np.unique(np.concatenate([idx, self_idx]))
        p, q, keep = oracle.site_frequencies(c.codes)
        ref = oracle.relatedness_pairs(c.codes, p, q, keep, np.stack([xs[idx], ys[idx]], 1))
        summary.append((c.name, compare(rows[idx], ref)))
    for name, s in summary:
        print(name, s)
    print({k: st[k] for k in ("gh_passes", "fp64_pairs", "waves", "slots", "nonconverged")})
