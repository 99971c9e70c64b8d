"""The oracle's restatement of the reference's default hard-call estimator
(conditional least squares with the Brier objective, src/coefficients.rs:166-278),
checked against an independent numpy evaluation of its parts.  CPU only."""
import numpy as np
import pytest

from kestrel_b200 import synth


def numpy_rows(p, q):
    """m[v, gx, gy, :] from the closed forms of src/iis.rs:279-462 for two alleles."""
    R = np.zeros((len(p), 3, 3, 9))
    for gx, t in ((0, p), (2, q)):
        R[:, gx, gx] = np.stack([t, t**2, t**2, t**3, t**2, t**3, t**2, t**3, t**4], 1)
    for gx, a, k in ((0, p, q), (2, q, p)):
        gy = 2 - gx
        R[:, gx, gy, 1] = a * k
        R[:, gx, gy, 3] = a * k**2
        R[:, gx, gy, 5] = a**2 * k
        R[:, gx, gy, 8] = a**2 * k**2
        R[:, gx, 1, 2] = a * k
        R[:, gx, 1, 3] = 2 * a**2 * k
        R[:, gx, 1, 7] = a**2 * k
        R[:, gx, 1, 8] = 2 * a**3 * k
    R[:, 1, 0, 4] = p * q
    R[:, 1, 0, 5] = 2 * p**2 * q
    R[:, 1, 0, 7] = p**2 * q
    R[:, 1, 0, 8] = 2 * p**3 * q
    R[:, 1, 2, 4] = p * q
    R[:, 1, 2, 5] = 2 * q**2 * p
    R[:, 1, 2, 7] = q**2 * p
    R[:, 1, 2, 8] = 2 * q**3 * p
    R[:, 1, 1, 6] = 2 * p * q
    R[:, 1, 1, 7] = p * q * (p + q)
    R[:, 1, 1, 8] = 4 * p**2 * q**2
    return R


def row_index(n, x, y):
    return x * n - x * (x - 1) // 2 + (y - x)


@pytest.fixture(scope="module")
def cohort():
    return synth.make_cohort(40, 4000, 11, missing=0.0,
                             planted={"parent_offspring": 4, "full_sib": 4}, name="cls")


def test_brier_and_kkt_against_numpy(oracle, cohort):
    codes = cohort.codes
    n, m = codes.shape
    out = oracle.cls_relatedness(codes, iterations=100)
    g = codes.astype(np.int64)
    p = (2 - g).sum(0) / (2 * n)
    q = g.sum(0) / (2 * n)
    R = numpy_rows(p, q)
    Q = np.einsum("vabi,vabj->ij", R, R) / m
    for x, y in [(0, 1), (2, 9), (7, 7), (13, 39), (20, 21)]:
        r = out[row_index(n, x, y)]
        assert r["x"] == x and r["y"] == y
        c = -R[np.arange(m), g[x], g[y]].sum(0) / m
        d = r["jacquard"]
        brier = d @ Q @ d + 2 * c @ d + 1
        assert abs(brier - r["obj"]) <= 1e-12 * abs(brier)
        if x != y and r["iters"] < 100:
            grad = Q @ d + c
            lam = d @ grad
            viol = np.where(d > 0, np.abs(grad - lam), np.maximum(lam - grad, 0))
            assert viol.max() < 1e-8


def test_self_pairs_use_delta1_and_delta7(oracle, cohort):
    out = oracle.cls_relatedness(cohort.codes)
    s = out[out["x"] == out["y"]]["jacquard"]
    assert np.allclose(s[:, 0] + s[:, 6], 1.0, atol=1e-12)
    assert np.all(s[:, [1, 2, 3, 4, 5, 7, 8]] == 0.0)


def test_incomplete_sites_are_dropped(oracle, cohort):
    codes = cohort.codes.copy()
    base = oracle.cls_relatedness(codes)
    extra = np.full((codes.shape[0], 3), 1, np.uint8)
    extra[5, 0] = synth.MISSING          # a missing call drops the whole site
    extra[0, 1] = synth.MISSING
    extra[:, 2] = synth.MISSING
    with_missing = oracle.cls_relatedness(np.concatenate([codes, extra], 1))
    assert np.array_equal(base["jacquard"], with_missing["jacquard"])
    assert np.array_equal(base["obj"], with_missing["obj"])


def test_supplied_frequencies(oracle, cohort):
    codes = cohort.codes
    n = codes.shape[0]
    g = codes.astype(np.int64)
    af = np.stack([(2 - g).sum(0) / (2 * n), g.sum(0) / (2 * n)], 1)
    a = oracle.cls_relatedness(codes)
    b = oracle.cls_relatedness(codes, af=af)
    assert np.array_equal(a["jacquard"], b["jacquard"])


def test_planted_recovery(oracle):
    c = synth.make_cohort(64, 10_000, 5, missing=0.0,
                          planted={"parent_offspring": 4, "full_sib": 4, "half_sib": 4}, name="cls")
    out = oracle.cls_relatedness(c.codes)
    n = c.codes.shape[0]
    for a, b, rel, _ in c.planted:
        d = out[row_index(n, a, b)]["jacquard"]
        if rel == "parent_offspring":
            assert d[7] > 0.85
        elif rel == "full_sib":
            assert 0.15 < d[6] < 0.4 and 0.3 < d[7] < 0.65
        else:
            assert 0.25 < d[7] < 0.7 and d[8] > 0.3


def test_num_samples_and_iteration_cap(oracle, cohort):
    full = oracle.cls_relatedness(cohort.codes)
    sub = oracle.cls_relatedness(cohort.codes, num_samples=10)
    n = cohort.codes.shape[0]
    for r in sub:
        ref = full[row_index(n, int(r["x"]), int(r["y"]))]
        assert np.array_equal(r["jacquard"], ref["jacquard"])
    capped = oracle.cls_relatedness(cohort.codes, iterations=2)
    assert capped["iters"].max() <= 2


# ---- tri- and tetra-allelic sites (the reference's gt3 / gt4)

def table_row(i, j, k, l, f):
    """The nine conditional probabilities of genotypes (i, j), (k, l) (i <= j,
    k <= l) from the closed forms of src/iis.rs:279-462, the mode chosen by the
    allele equalities as src/iis.rs:76-118 does."""
    pi, pj, pk, pl = f[i], f[j], f[k], f[l]
    eq = (i == j, i == k, i == l, j == k, j == l, k == l)
    r = np.zeros(9)
    if all(eq):                                           # ii-ii
        r[:] = [pi, pi**2, pi**2, pi**3, pi**2, pi**3, pi**2, pi**3, pi**4]
    elif eq == (1, 0, 0, 0, 0, 1):                        # ii-kk
        r[[1, 3, 5, 8]] = [pi * pk, pi * pk**2, pi**2 * pk, pi**2 * pk**2]
    elif eq in ((1, 1, 0, 1, 0, 0), (1, 0, 1, 0, 1, 0)):  # ii-il, ii-ki
        o = pl if eq[1] else pk
        r[[2, 3, 7, 8]] = [pi * o, 2 * pi**2 * o, pi**2 * o, 2 * pi**3 * o]
    elif eq == (1, 0, 0, 0, 0, 0):                        # ii-kl
        r[[3, 8]] = [2 * pi * pk * pl, 2 * pi**2 * pk * pl]
    elif eq == (0, 1, 1, 0, 0, 1):                        # ij-ii
        r[[4, 5, 7, 8]] = [pi * pj, 2 * pi**2 * pj, pi**2 * pj, 2 * pi**3 * pj]
    elif eq == (0, 0, 0, 1, 1, 1):                        # ij-jj
        r[[4, 5, 7, 8]] = [pi * pj, 2 * pj**2 * pi, pj**2 * pi, 2 * pj**3 * pi]
    elif eq == (0, 0, 0, 0, 0, 1):                        # ij-kk
        r[[5, 8]] = [2 * pi * pj * pk, 2 * pk**2 * pi * pj]
    elif eq in ((0, 1, 0, 0, 1, 0), (0, 0, 1, 1, 0, 0)):  # ij-ij, ij-ji
        r[[6, 7, 8]] = [2 * pi * pj, pi * pj * (pi + pj), 4 * pi**2 * pj**2]
    elif eq == (0, 1, 0, 0, 0, 0):                        # ij-il
        r[[7, 8]] = [pi * pj * pl, 4 * pi**2 * pj * pl]
    elif eq == (0, 0, 1, 0, 0, 0):                        # ij-ki
        r[[7, 8]] = [pi * pj * pk, 4 * pi**2 * pj * pk]
    elif eq == (0, 0, 0, 1, 0, 0):                        # ij-jl
        r[[7, 8]] = [pi * pj * pl, 4 * pi * pj**2 * pl]
    elif eq == (0, 0, 0, 0, 1, 0):                        # ij-kj
        r[[7, 8]] = [pi * pj * pk, 4 * pi * pj**2 * pk]
    elif eq == (0, 0, 0, 0, 0, 0):                        # ij-kl
        r[8] = 4 * pi * pj * pk * pl
    else:
        raise AssertionError(eq)
    return r


def alleles_of(g):
    b = 0
    while (b + 1) * (b + 2) // 2 <= g:
        b += 1
    return g - b * (b + 1) // 2, b


def table_rows(freq, n_alleles):
    ng = n_alleles * (n_alleles + 1) // 2
    R = np.zeros((ng, ng, 9))
    for gx in range(ng):
        for gy in range(ng):
            R[gx, gy] = table_row(*alleles_of(gx), *alleles_of(gy), freq)
    return R


def test_iis_rows_match_the_closed_forms(oracle):
    rng = np.random.default_rng(3)
    for _ in range(20):
        f = rng.dirichlet(np.ones(4))
        R = table_rows(f, 4)
        for gx in range(10):
            for gy in range(10):
                got = oracle.iis_row(gx, gy, f)
                assert np.allclose(got, R[gx, gy], rtol=1e-14, atol=1e-300), (gx, gy)
    # two alleles: the biallelic rows
    p = rng.uniform(0.05, 0.95, 50)
    B = numpy_rows(p, 1 - p)
    for v in range(50):
        for gx in range(3):
            for gy in range(3):
                assert np.allclose(oracle.iis_row(gx, gy, [p[v], 1 - p[v]]), B[v, gx, gy], rtol=1e-14)


def test_tri_site_with_an_absent_allele_is_biallelic(oracle, cohort):
    codes = cohort.codes
    n = codes.shape[0]
    base = oracle.cls_relatedness(codes)
    g = codes.astype(np.int64)
    p = (2 - g).sum(0) / (2 * n)
    cut = 3000
    mg = codes[:, cut:].copy()        # 0/0, 0/1, 1/1 keep their index with three alleles
    al = np.full(mg.shape[1], 3, np.uint8)
    for maf in (None, np.stack([p[cut:], 1 - p[cut:], 0 * p[cut:], 0 * p[cut:]], 1)):
        out = oracle.cls_relatedness(codes[:, :cut], multi=(mg, al, maf))
        assert np.abs(out["jacquard"] - base["jacquard"]).max() < 1e-9
        assert np.abs(out["obj"] - base["obj"]).max() < 1e-12
        assert np.mean(out["iters"] == base["iters"]) > 0.99


def test_multi_allelic_brier_and_kkt_against_numpy(oracle, cohort):
    codes = cohort.codes[:, :1500]
    n, m = codes.shape
    mg, al = synth.make_multiallelic(n, 300, 5)
    mg[3, 7] = 255                          # a missing call drops site 7
    out = oracle.cls_relatedness(codes, multi=(mg, al, None))
    g = codes.astype(np.int64)
    p = (2 - g).sum(0) / (2 * n)
    Rb = numpy_rows(p, 1 - p)
    keep = [v for v in range(mg.shape[1]) if v != 7]
    Rm = []
    for v in keep:
        cnt = np.zeros(4)
        for s in range(n):
            a, b = alleles_of(mg[s, v])
            cnt[a] += 1
            cnt[b] += 1
        Rm.append(table_rows(cnt / (2 * n), al[v]))
    M = m + len(keep)
    Q = np.einsum("vabi,vabj->ij", Rb, Rb) + sum(np.einsum("abi,abj->ij", R, R) for R in Rm)
    Q /= M
    for x, y in [(0, 1), (2, 9), (7, 7), (13, 39), (20, 21)]:
        r = out[row_index(n, x, y)]
        c = Rb[np.arange(m), g[x], g[y]].sum(0) + sum(R[mg[x, v], mg[y, v]] for R, v in zip(Rm, keep))
        c = -c / M
        d = r["jacquard"]
        brier = d @ Q @ d + 2 * c @ d + 1
        assert abs(brier - r["obj"]) <= 1e-11 * abs(brier)
        if x != y and r["iters"] < 100:
            grad = Q @ d + c
            lam = d @ grad
            viol = np.where(d > 0, np.abs(grad - lam), np.maximum(lam - grad, 0))
            assert viol.max() < 1e-8
