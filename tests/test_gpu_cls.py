"""GPU parity of the CLS/Brier hard-call estimator (kg_relatedness_gt, the
reference's default -f GT path, src/coefficients.rs:166-278) against the FP64
oracle.  Same bar as the ML path (tests/parity.py): Delta and kinship within
1e-5 absolute and the Brier objective within 1e-6 relative wherever the
oracle's log10 cond is below 15, and the condition flag equal there."""
import numpy as np
import pytest

import kestrel_b200 as kb
from kestrel_b200 import synth

from .parity import check_values, compare

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def est():
    e = kb.Estimator()
    yield e
    e.close()


@pytest.fixture(scope="module")
def complete():
    return synth.make_cohort(64, 10_000, 21, missing=0.0,
                             planted={"parent_offspring": 4, "full_sib": 4, "half_sib": 4,
                                      "first_cousin": 4}, name="cls")


@pytest.mark.parametrize("precision", ["fp32c", "fp64"])
def test_cls_parity(est, oracle, complete, precision):
    ref = oracle.cls_relatedness(complete.codes)
    est.set_precision(precision)
    est.load(complete.codes)
    gpu = est.relatedness_gt()
    est.set_precision("fp32c")
    stats = compare(gpu, ref)
    same_iters = float(np.mean(gpu["iters"] == ref["iters"]))
    print(precision, stats, "same QP iterations", same_iters)
    assert same_iters > 0.95
    s = gpu[gpu["x"] == gpu["y"]]["jacquard"]
    assert np.allclose(s[:, 0] + s[:, 6], 1.0, atol=1e-9)
    assert np.all(s[:, [1, 2, 3, 4, 5, 7, 8]] == 0.0)


def test_cls_drops_incomplete_sites(est, oracle):
    c = synth.make_cohort(48, 20_000, 22, missing=0.0005, name="cls-miss")
    complete_sites = int(np.all(c.codes < 3, 0).sum())
    assert 0 < complete_sites < c.codes.shape[1]
    ref = oracle.cls_relatedness(c.codes)
    est.load(c.codes)
    gpu = est.relatedness_gt()
    compare(gpu, ref)


def test_cls_supplied_frequencies_and_subset(est, oracle, complete):
    codes = complete.codes
    n = codes.shape[0]
    rng = np.random.default_rng(4)
    p = np.clip(rng.uniform(0.05, 0.95, codes.shape[1]), 0.05, 0.95)
    af = np.stack([p, 1.0 - p], 1)
    ref = oracle.cls_relatedness(codes, af=af, num_samples=40)
    est.load(codes, allele_frequencies=af)
    gpu = est.relatedness_gt(num_samples=40)
    compare(gpu, ref)
    est.load(codes)


def test_cls_iteration_cap(est, oracle, complete):
    ref = oracle.cls_relatedness(complete.codes, iterations=3)
    est.load(complete.codes)
    gpu = est.relatedness_gt(iterations=3)
    assert gpu["iters"].max() <= 3
    assert np.mean(gpu["iters"] == ref["iters"]) > 0.95


def test_cls_no_complete_site(est):
    codes = np.ones((8, 64), np.uint8)
    codes[np.arange(8), np.arange(8)] = synth.MISSING
    codes[:, 8:] = synth.MISSING
    est.load(codes)
    with pytest.raises(kb.KestrelError) as e:
        est.relatedness_gt()
    assert e.value.status == kb.KG_ENOSITES


# ---- tri- and tetra-allelic sites (kg_load_multiallelic)

@pytest.fixture(scope="module")
def multi(complete):
    g, al = synth.make_multiallelic(complete.codes.shape[0], 700, 23)
    g[5, 11] = 255                       # a missing call drops site 11
    return g, al


def test_cls_multiallelic_parity(est, oracle, complete, multi):
    g, al = multi
    ref = oracle.cls_relatedness(complete.codes, multi=(g, al, None))
    est.load(complete.codes)
    est.load_multiallelic(g, al)
    gpu = est.relatedness_gt()
    stats = compare(gpu, ref)
    same_iters = float(np.mean(gpu["iters"] == ref["iters"]))
    print(stats, "same QP iterations", same_iters)
    assert same_iters > 0.95
    # without them the result changes, and loading genotypes again clears them
    est.load(complete.codes)
    plain = est.relatedness_gt()
    assert np.abs(plain["jacquard"] - gpu["jacquard"]).max() > 1e-6
    compare(plain, oracle.cls_relatedness(complete.codes))


def test_cls_multiallelic_supplied_frequencies_and_subset(est, oracle, complete, multi):
    g, al = multi
    rng = np.random.default_rng(8)
    maf = np.zeros((g.shape[1], 4))
    for v in range(g.shape[1]):
        maf[v, :al[v]] = rng.dirichlet(np.ones(al[v]))
    ref = oracle.cls_relatedness(complete.codes, num_samples=40, multi=(g, al, maf))
    est.load(complete.codes)
    est.load_multiallelic(g, al, maf)
    gpu = est.relatedness_gt(num_samples=40)
    compare(gpu, ref)


def test_cls_tri_site_with_an_absent_allele_is_biallelic(est, complete):
    codes = complete.codes
    est.load(codes)
    base = est.relatedness_gt()
    cut = 7000
    est.load(codes[:, :cut])
    est.load_multiallelic(codes[:, cut:], np.full(codes.shape[1] - cut, 3, np.uint8))
    split = est.relatedness_gt()
    # the same estimator up to where the sums run (FP32 moments vs FP64 rows),
    # within the parity bar
    print(check_values(split["jacquard"], split["obj"], np.log10(split["cond"]), base))


def test_cls_multiallelic_bad_index(est, complete):
    g = np.zeros((complete.codes.shape[0], 4), np.uint8)
    g[2, 1] = 6                          # index 6 needs four alleles
    est.load(complete.codes)
    est.load_multiallelic(g, np.full(4, 3, np.uint8))
    with pytest.raises(kb.KestrelError) as e:
        est.relatedness_gt()
    assert e.value.status == kb.KG_EINVAL
    est.load(complete.codes)


def test_python_gt_api_routes_multiallelic_sites(oracle, complete, multi):
    g, al = multi
    n = complete.codes.shape[0]
    # allele pairs: biallelic sites from the codes, the others from the indices
    bi = np.stack([(complete.codes >= 1).astype(np.uint8), (complete.codes >= 2).astype(np.uint8)], 2)
    mj = np.zeros(g.shape, np.int64)
    for k in range(1, 4):
        mj += g >= k * (k + 1) // 2
    mi = g.astype(np.int64) - mj * (mj + 1) // 2
    ma = np.stack([mi, mj], 2).astype(np.uint8)
    ma[g == 255] = 255
    # the allele count of a site is its largest called allele + 1 here
    top = np.where(g == 255, 0, mj).max(0)
    keep = top >= 2
    genotypes = np.concatenate([bi.transpose(1, 0, 2), ma[:, keep].transpose(1, 0, 2)], 0)
    co = kb.relatedness_coefficients_gt(genotypes, estimator="cls")
    ref = oracle.cls_relatedness(complete.codes, multi=(g[:, keep], (top[keep] + 1).astype(np.uint8), None))
    x, y = ref["x"].astype(int), ref["y"].astype(int)
    lc = np.log10(ref["cond"])
    below = np.isfinite(lc) & (lc < 15)
    assert np.abs(co.jacquard[x, y] - ref["jacquard"]).max(1)[below].max() <= 1e-5
    assert co.jacquard.shape == (n, n, 9)
