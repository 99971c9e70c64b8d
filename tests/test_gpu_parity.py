"""GPU parity of the CUDA path (through the C ABI) against the FP64 oracle.

Tolerances (the estimator's stated bar, tests/parity.py): Delta and kinship
within 1e-5 absolute and the objective within 1e-6 relative wherever the
oracle's log10 cond is below 15, and the condition flag (log10 cond > 15)
equal there."""
import numpy as np
import pytest

import kestrel_b200 as kb
from kestrel_b200 import synth

from .parity import compare

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def est():
    e = kb.Estimator()
    yield e
    e.close()


@pytest.mark.parametrize("precision", ["fp32c", "fp64"])
def test_config0_all_pairs(est, oracle, cfg0, precision):
    ref = oracle.relatedness(cfg0.codes)
    est.set_precision(precision)
    est.load(cfg0.codes)
    gpu = est.relatedness()
    stats = compare(gpu, ref)
    print(precision, stats, est.run_stats())
    if precision == "fp64":
        # FP64 follows the reference's iteration path
        assert np.mean(gpu["iters"] == ref["iters"]) > 0.97
    est.set_precision("fp32c")


def test_config1_sampled_pairs(est, oracle):
    c = synth.config1(n_samples=256, n_sites=100_000)
    est.load(c.codes)
    gpu = est.relatedness()
    p, q, keep = oracle.site_frequencies(c.codes)
    rng = np.random.default_rng(3)
    idx = rng.choice(len(gpu), 300, replace=False)
    planted = {(a, b) for a, b, _, _ in c.planted}
    xs, ys = gpu["x"].astype(int), gpu["y"].astype(int)
    extra = [i for i in range(len(gpu)) if (xs[i], ys[i]) in planted]
    idx = np.unique(np.concatenate([idx, extra]))
    ref = oracle.relatedness_pairs(c.codes, p, q, keep, np.stack([xs[idx], ys[idx]], 1))
    print(compare(gpu[idx], ref))


def test_num_samples_maf_and_af(est, oracle):
    c = synth.make_cohort(48, 5000, seed=21)
    est.load(c.codes)
    gpu = est.relatedness(num_samples=20, maf=0.1)
    ref = oracle.relatedness(c.codes, num_samples=20, maf=0.1)
    compare(gpu, ref)
    af = np.stack([c.p_true, 1 - c.p_true], 1)
    est.load(c.codes, allele_frequencies=af)
    gpu = est.relatedness(num_samples=12)
    ref = oracle.relatedness(c.codes, af=af, num_samples=12)
    compare(gpu, ref)


def test_ragged_small_cases(est, oracle):
    """Tiny cohorts crossing word and segment edges (M = 1..70, 2047..2049)."""
    for seed, (n, m) in enumerate([(3, 1), (4, 31), (5, 33), (6, 70), (3, 2047), (3, 2049), (7, 4100)]):
        c = synth.make_cohort(n, m, seed=100 + seed, missing=0.0)
        p, q, keep = oracle.site_frequencies(c.codes)
        if keep.sum() == 0:
            continue
        est.load(c.codes)
        try:
            ref = oracle.relatedness(c.codes)
        except RuntimeError:
            continue
        gpu = est.relatedness()
        compare(gpu, ref)


def test_pair_without_sites_is_reported(est):
    codes = np.array([[0, 1, 2, 3, 3], [3, 3, 3, 0, 1], [1, 1, 0, 2, 0]], np.uint8)
    est.load(codes)
    with pytest.raises(kb.KestrelError) as ei:
        est.relatedness()
    assert ei.value.status == 5
    rows = est.relatedness(allow_nosites=True)
    bad = np.isnan(rows["obj"])
    assert bad.sum() == 1 and rows["x"][bad][0] == 0 and rows["y"][bad][0] == 1


def test_bad_codes_rejected(est):
    codes = np.array([[0, 1, 7], [1, 1, 0]], np.uint8)
    est.load(codes)
    with pytest.raises(kb.KestrelError):
        est.relatedness()


def test_batch_matches_single_runs(est, oracle):
    cohorts = synth.config2(scale=0.05)
    outs = est.relatedness_batch([(c.codes,) for c in cohorts])
    for c, out in zip(cohorts, outs):
        est.load(c.codes)
        single = est.relatedness()
        np.testing.assert_array_equal(out["jacquard"], single["jacquard"])
        np.testing.assert_array_equal(out["obj"], single["obj"])
    for c, out in zip(cohorts, outs):          # every cohort of the batch, every pair
        compare(out, oracle.relatedness(c.codes))
    # the same call into caller-owned row buffers, filled in place
    bufs = [np.zeros(len(o) + 3, kb.OUTPUT_DTYPE) for o in outs]
    again = est.relatedness_batch([(c.codes,) for c in cohorts], out=bufs)
    for o, a, b in zip(outs, again, bufs):
        assert a is b
        np.testing.assert_array_equal(b[:len(o)].view(np.uint8), o.view(np.uint8))


def test_python_api_build_arrays(oracle, cfg0):
    g = np.zeros((cfg0.n_sites, cfg0.n_samples, 2), np.uint8)
    codes = cfg0.codes.T
    g[..., 0] = (codes >= 1) & (codes != 3)
    g[..., 1] = (codes == 2)
    g[codes == 3] = 255
    co = kb.relatedness_coefficients_gt(g)
    ref = oracle.relatedness(cfg0.codes)
    jac, kin, inb = kb.build_arrays(ref, cfg0.n_samples)
    assert np.abs(co.kinship - kin).max() < 1e-5
    assert np.abs(co.inbreeding - inb).max() < 1e-5
    perm = [0, 1, 4, 5, 2, 3, 6, 7, 8]
    np.testing.assert_allclose(co.jacquard[3, 9], co.jacquard[9, 3][perm])


def test_config1_full_size_sampled_pairs(est, oracle):
    """The benchmark's own workload, N=1024 x M=100,000 (523,776 pairs + 1,024
    self): 200 random pairs and every planted pair against the oracle, and the
    size-independent properties of all rows (Delta on the simplex, finite
    objective, kinship in [0, 1], planted relationships recovered)."""
    c = synth.config1()
    est.load(c.codes)
    gpu = est.relatedness()
    n = c.codes.shape[0]
    assert len(gpu) == n * (n + 1) // 2
    jac = gpu["jacquard"]
    assert np.all(jac >= 0.0) and np.abs(jac.sum(1) - 1.0).max() < 1e-12
    assert np.all(np.isfinite(gpu["obj"]))
    kin = jac @ kb.KINSHIP_VECTOR
    assert kin.min() >= 0.0 and kin.max() <= 1.0 + 1e-12
    xs, ys = gpu["x"].astype(int), gpu["y"].astype(int)
    pos = {(a, b): i for i, (a, b) in enumerate(zip(xs, ys))}
    for a, b, rel, delta in c.planted:
        i = pos[(a, b)]
        assert np.abs(kin[i] - delta @ kb.KINSHIP_VECTOR) < 0.05, (rel, kin[i])
    rng = np.random.default_rng(11)
    idx = rng.choice(len(gpu), 200, replace=False)
    idx = np.unique(np.concatenate([idx, [pos[(a, b)] for a, b, _, _ in c.planted]]))
    p, q, keep = oracle.site_frequencies(c.codes)
    ref = oracle.relatedness_pairs(c.codes, p, q, keep, np.stack([xs[idx], ys[idx]], 1))
    print(compare(gpu[idx], ref), est.run_stats()["nonconverged"])


def test_config0_against_committed_golden_rows(est):
    """The CUDA path on the committed config-0 genotypes against the committed
    oracle rows (no live oracle run)."""
    import os
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "config0_oracle.npz"))
    ref = np.zeros(len(g["x"]), kb.OUTPUT_DTYPE)
    for k in ("x", "y", "jacquard", "obj", "iters", "cond"):
        ref[k] = g[k]
    est.load(g["codes"])
    print(compare(est.relatedness(), ref))
