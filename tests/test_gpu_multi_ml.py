"""GPU parity of the maximum-likelihood estimator with tri- and tetra-allelic
sites (kg_load_multiallelic + kg_relatedness) against the oracle's GL/PL path
on the same calls as one-hot likelihoods (kor_gl_relatedness: the per-site
allele-frequency fit for 2-4 alleles, the maf cut, zero-frequency alleles
dropped as in src/wrapper.rs:349-409, rows sum over genotype pairs of GLx GLy
m, src/coefficients.rs:99-106).  The bar of tests/parity.py."""
import numpy as np
import pytest

import kestrel_b200 as kb
from kestrel_b200 import synth

from .parity import compare
from .test_oracle_gl import one_hot

pytestmark = pytest.mark.gpu


def one_hot_multi(g, al):
    """Genotype indices [samples, sites] (255 = missing) and allele counts ->
    one-hot likelihoods [sites, samples, G] of the tri- and of the
    tetra-allelic sites, NaN where missing."""
    out = []
    for a in (3, 4):
        sel = np.nonzero(al == a)[0]
        ng = a * (a + 1) // 2
        gl = np.zeros((len(sel), g.shape[0], ng))
        sub = g[:, sel].T
        for k in range(ng):
            gl[..., k] = sub == k
        gl[sub == 255] = np.nan
        out.append(gl if len(sel) else None)
    return out


@pytest.fixture(scope="module")
def cohort():
    co = synth.make_cohort(40, 3000, 81, missing=0.02, planted={"parent_offspring": 3, "full_sib": 3},
                           name="multi-ml")
    g, al = synth.make_multiallelic(40, 500, 82, missing=0.02)
    return co, g, al


@pytest.fixture(scope="module")
def est():
    e = kb.Estimator()
    yield e
    e.close()


def _oracle(oracle, co, g, al, **kw):
    gl3, gl4 = one_hot_multi(g, al)
    rows, af = oracle.gl_relatedness(one_hot(co.codes), gl3=gl3, gl4=gl4, **kw)
    return rows, af


def test_multiallelic_sites_parity(est, oracle, cohort):
    co, g, al = cohort
    ref, af = _oracle(oracle, co, g, al)
    est.load(co.codes)
    est.load_multiallelic(g, al)
    gpu = est.relatedness()
    st = est.run_stats()
    print(compare(gpu, ref), st["sites_used"], st["sites_discarded"])
    # the oracle's frequencies come grouped: biallelic, tri-, tetra-allelic
    n2, n3 = co.codes.shape[1], int(np.sum(al == 3))
    nz = (af > 0).sum(1)
    assert st["sites_used"] == [int(np.sum(nz == 2)), int(np.sum(nz == 3)), int(np.sum(nz == 4))]
    # the cohort exercises every branch: multi-allelic sites cut to fewer
    # alleles (a rare allele below maf, whose carriers get zero rows)
    assert st["sites_used"][1] > 0 and st["sites_used"][2] > 0
    assert np.any(nz[n2:n2 + n3] == 2) and np.any(nz[n2 + n3:] < 4)
    # and they change the estimate
    est.load(co.codes)
    bi = est.relatedness()
    assert np.abs(bi["jacquard"] - gpu["jacquard"]).max() > 1e-4


def test_multiallelic_subset_maf_and_cap(est, oracle, cohort):
    co, g, al = cohort
    ref, _ = _oracle(oracle, co, g, al, maf=0.05, num_samples=25)
    est.load(co.codes)
    est.load_multiallelic(g, al)
    gpu = est.relatedness(num_samples=25, maf=0.05)
    compare(gpu, ref)
    ref5, _ = _oracle(oracle, co, g, al, iterations=5)
    gpu5 = est.relatedness(iterations=5)
    assert gpu5["iters"].max() <= 5
    ok = ref5["iters"] < 5
    lc = np.log10(ref5["cond"])
    d = np.abs(gpu5["jacquard"] - ref5["jacquard"]).max(1)
    assert d[ok & np.isfinite(lc) & (lc < 15)].max() <= 1e-5


def test_tri_site_with_an_absent_allele_is_biallelic(est, cohort):
    """Biallelic calls given as tri-allelic sites whose third allele nobody
    carries: the fit gives it frequency 0, the site keeps two alleles, and the
    estimate equals the all-biallelic one (generic rows against the closed
    forms: within the bar)."""
    co, _, _ = cohort
    cut = 2000
    codes = co.codes
    # maf off the 1 / (2 N) tie: a fully called singleton's fitted frequency
    # sits within the fit's tolerance of it, in two and in three dimensions
    est.load(codes)
    base = est.relatedness(maf=0.01)
    est.load(codes[:, :cut])
    tri = codes[:, cut:].copy()                 # 0/0 = 0, 0/1 = 1, 1/1 = 2 in the VCF order too
    tri[tri == synth.MISSING] = 255
    est.load_multiallelic(tri, np.full(tri.shape[1], 3, np.uint8))
    split = est.relatedness(maf=0.01)
    assert est.run_stats()["sites_used"][1] == 0
    print(compare(split, base))


def test_host_driven_waves_equal_device_loop(est, cohort, monkeypatch):
    co, g, al = cohort
    est.load(co.codes)
    est.load_multiallelic(g, al)
    a = est.relatedness()
    monkeypatch.setenv("KESTREL_HOST_WAVES", "1")
    b = est.relatedness()
    assert np.array_equal(a.view(np.uint8), b.view(np.uint8))


def _multi_pl_records(g, al):
    """VCF lines of tri- and tetra-allelic sites with one-hot PL (0 at the
    call, 255 elsewhere; '.' when missing), in the loaded order."""
    alts = {3: "C,G", 4: "C,G,T"}
    lines = []
    for v in range(g.shape[1]):
        ng = int(al[v]) * (int(al[v]) + 1) // 2
        calls = []
        for s in range(g.shape[0]):
            if g[s, v] == 255:
                calls.append(".")
                continue
            pl = ["255"] * ng
            pl[int(g[s, v])] = "0"
            calls.append(",".join(pl))
        lines.append(f"3\t{v + 1}\t.\tA\t{alts[int(al[v])]}\t.\tPASS\t.\tPL\t" + "\t".join(calls))
    return lines


def test_cli_pl_with_multiallelic_records_matches_oracle(oracle, cohort):
    import os
    import subprocess
    import tempfile
    from .test_gpu_workloads import _read_tsv, _tsv_values
    from .parity import check_values
    co, g, al = cohort
    ref, af = _oracle(oracle, co, g, al, num_samples=30)
    nz = (af > 0).sum(1)
    cli = os.path.join(os.path.dirname(kb.__file__), "bin", "kestrel")
    with tempfile.TemporaryDirectory() as td:
        vcf = os.path.join(td, "in.vcf")
        tsv = os.path.join(td, "out.tsv")
        synth.write_vcf(vcf, co.codes, field="PL")
        with open(vcf, "a") as fh:
            fh.write("\n".join(_multi_pl_records(g, al)) + "\n")
        r = subprocess.run([cli, vcf, tsv, "-f", "PL", "-s", "30"], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        _, rows = _read_tsv(tsv)
    assert f"Found {int(np.sum(al == 3))} tri-allelic sites" in r.stderr
    assert f"Found {int(np.sum(al == 4))} tetra-allelic sites" in r.stderr
    assert f"Identified {int(np.sum(nz == 2))} di-allelic sites" in r.stderr
    assert f"Identified {int(np.sum(nz == 3))} tri-allelic sites" in r.stderr
    assert f"Identified {int(np.sum(nz == 4))} tetra-allelic sites" in r.stderr
    assert f"Discarded {int(np.sum(nz < 2))} non-segregating sites" in r.stderr
    assert len(rows) == len(ref)
    print(check_values(*_tsv_values(rows), ref))


def test_python_gt_api_ml_routes_multiallelic_sites(oracle, cohort):
    co, g, al = cohort
    bi = np.stack([(co.codes >= 1) & (co.codes != 3), co.codes == 2], 2).astype(np.uint8)
    bi[co.codes == 3] = 255
    mj = np.zeros(g.shape, np.int64)
    for k in range(1, 4):
        mj += g >= k * (k + 1) // 2
    mi = g.astype(np.int64) - mj * (mj + 1) // 2
    ma = np.stack([mi, mj], 2).astype(np.uint8)
    ma[g == 255] = 255
    # the API takes a site's allele count from its largest called allele
    top = np.where(g == 255, 0, mj).max(0)
    keep = top >= 2
    genotypes = np.concatenate([bi.transpose(1, 0, 2), ma[:, keep].transpose(1, 0, 2)], 0)
    res = kb.relatedness_coefficients_gt(genotypes, estimator="ml")
    ref, _ = _oracle(oracle, co, g[:, keep], (top[keep] + 1).astype(np.uint8))
    x, y = ref["x"].astype(int), ref["y"].astype(int)
    lc = np.log10(ref["cond"])
    below = np.isfinite(lc) & (lc < 15)
    assert np.abs(res.jacquard[x, y] - ref["jacquard"]).max(1)[below].max() <= 1e-5
