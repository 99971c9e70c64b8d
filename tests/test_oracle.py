"""CPU tests of the FP64 oracle (the checker): pinned against an independent
numpy restatement, known relationships and the swap symmetry of the reference."""
import numpy as np
import pytest

from kestrel_b200 import synth
from tests import npref


def test_allele_counts_match_numpy(oracle, cfg0):
    rc, oc = oracle.allele_counts(cfg0.codes)
    c = cfg0.codes
    obs = c != 3
    assert np.array_equal(oc, obs.sum(0))
    assert np.array_equal(rc, np.where(obs, 2 - c.astype(int), 0).sum(0))


def test_site_frequencies_are_the_allele_sqp(oracle, cfg0):
    # the reference's GL path fits each site's frequencies by an SQP
    # (src/allele/mod.rs); on hard calls its optimum is the count frequency
    # moved by the eps inside the log (about 5e-9), and it equals the fit on
    # one-hot likelihoods
    p, q, keep = oracle.site_frequencies(cfg0.codes, maf=0.0)
    rc, oc = oracle.allele_counts(cfg0.codes)
    x0 = rc / (2.0 * oc)
    assert np.abs(p - x0)[keep].max() < 1e-6      # the SQP stops at KKT tolerance 1e-8
    assert np.array_equal(keep, (x0 > 0) & (x0 < 1))
    codes = cfg0.codes
    gl = np.zeros(codes.T.shape + (3,))
    for g in range(3):
        gl[..., g] = codes.T == g
    gl[codes.T == 3] = np.nan
    af = oracle.gl_allele_frequencies(gl, maf=0.0)
    assert np.abs(af[:, 0] - p)[keep].max() < 1e-8     # per class vs per sample sums: the same fit


def test_maf_zeroing_drops_rare_sites(oracle):
    codes = np.zeros((10, 4), np.uint8)
    codes[0, 1] = 1          # one ALT allele out of 20 -> q = 0.05
    codes[:5, 2] = 1          # q = 0.25
    codes[:, 3] = 2           # monomorphic ALT
    p, q, keep = oracle.site_frequencies(codes, maf=0.1)
    assert list(keep) == [False, False, True, False]
    # default maf 1/(2N) = 0.05: the fitted q of the singleton lands about
    # 5e-9 below its count frequency 0.05, so the cut takes it, as the
    # reference's GL path does
    p, q, keep = oracle.site_frequencies(codes)
    assert list(keep) == [False, False, True, False]
    p, q, keep = oracle.site_frequencies(codes, maf=0.04)
    assert list(keep) == [False, True, True, False]


@pytest.mark.parametrize("delta_kind", ["uniform", "unrelated", "po", "random"])
def test_fgh_matches_independent_numpy(oracle, cfg0, delta_kind):
    p, q, keep = oracle.site_frequencies(cfg0.codes)
    rng = np.random.default_rng(7)
    delta = {"uniform": np.full(9, 1 / 9), "unrelated": np.eye(9)[8],
             "po": np.eye(9)[7], "random": rng.dirichlet(np.ones(9))}[delta_kind]
    for x, y in [(0, 1), (3, 3), (10, 40)]:
        f, g, H, n = oracle.eval_pair(cfg0.codes[x], cfg0.codes[y], p, q, keep, delta)
        fr, gr, Hr, nr = npref.fgh(cfg0.codes[x], cfg0.codes[y], p, q, keep, delta)
        assert n == nr
        assert abs(f - fr) <= 1e-12 * abs(fr)
        np.testing.assert_allclose(g, gr, rtol=1e-11, atol=1e-11)
        np.testing.assert_allclose(H, Hr, rtol=1e-10, atol=1e-9)


def test_planted_relationships_recovered(oracle):
    c = synth.make_cohort(40, 20_000, seed=11,
                          planted={"parent_offspring": 2, "full_sib": 2, "half_sib": 2,
                                   "first_cousin": 2})
    p, q, keep = oracle.site_frequencies(c.codes)
    pairs = [(a, b) for a, b, _, _ in c.planted]
    out = oracle.relatedness_pairs(c.codes, p, q, keep, pairs)
    for (a, b, rel, d), o in zip(c.planted, out):
        kin_true = d @ np.array([1, 0, .5, 0, .5, 0, .5, .25, 0])
        kin = o["jacquard"] @ np.array([1, 0, .5, 0, .5, 0, .5, .25, 0])
        assert abs(kin - kin_true) < 0.02, (rel, o["jacquard"])
        assert np.all(o["jacquard"] >= 0) and abs(o["jacquard"].sum() - 1) < 1e-12


def test_swap_symmetry(oracle, cfg0):
    """(y, x) equals (x, y) with D3<->D5 and D4<->D6 (src/lib.rs:138-149)."""
    p, q, keep = oracle.site_frequencies(cfg0.codes)
    pairs = [(1, 2), (5, 30), (12, 63)]
    a = oracle.relatedness_pairs(cfg0.codes, p, q, keep, pairs)
    b = oracle.relatedness_pairs(cfg0.codes, p, q, keep, [(y, x) for x, y in pairs])
    perm = [0, 1, 4, 5, 2, 3, 6, 7, 8]
    np.testing.assert_allclose(a["jacquard"], b["jacquard"][:, perm], atol=1e-7)
    np.testing.assert_allclose(a["obj"], b["obj"], rtol=1e-12)


def test_full_config0_runs_and_is_feasible(oracle, cfg0):
    out = oracle.relatedness(cfg0.codes)
    n = cfg0.n_samples
    assert len(out) == n * (n + 1) // 2
    assert np.all(out["jacquard"] >= 0)
    np.testing.assert_allclose(out["jacquard"].sum(1), 1.0, atol=1e-12)
    assert np.all(out["iters"] < 100)
    # order: x ascending, y = x..n-1 (src/coefficients.rs:77-136)
    xs, ys = np.triu_indices(n)
    assert np.array_equal(out["x"], xs) and np.array_equal(out["y"], ys)
    # self pairs of outbred samples: Delta7 dominates
    self_rows = out[out["x"] == out["y"]]
    assert np.all(self_rows["jacquard"][:, 6] > 0.9)


def test_no_jointly_observed_site_is_an_error(oracle):
    codes = np.array([[0, 1, 2, 3, 3], [3, 3, 3, 0, 1], [1, 1, 0, 2, 0]], np.uint8)
    with pytest.raises(RuntimeError):
        oracle.relatedness(codes)


def _golden():
    import os
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "config0_oracle.npz"))
    return {k: g[k] for k in g.files}


def test_oracle_reproduces_committed_golden_rows(oracle):
    """The oracle on the committed config-0 genotypes gives the committed rows
    (tests/golden/make_golden.py), to the last few ulps across hosts."""
    g = _golden()
    rows = oracle.relatedness(g["codes"])
    assert np.array_equal(rows["x"], g["x"]) and np.array_equal(rows["y"], g["y"])
    assert np.array_equal(rows["iters"], g["iters"])
    assert np.abs(rows["jacquard"] - g["jacquard"]).max() <= 1e-12
    assert (np.abs(rows["obj"] - g["obj"]) / np.abs(g["obj"])).max() <= 1e-12
