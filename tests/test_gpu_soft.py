"""GPU parity of the GL/PL estimator on soft genotype likelihoods
(kg_relatedness_gl, src/wrapper.rs:89-330) against the oracle's restatement
(kor_gl_relatedness), with the same bar as the hard-call path."""
import numpy as np
import pytest

import kestrel_b200 as kb
from kestrel_b200 import synth

from .parity import compare
from .test_oracle_gl import one_hot, soft_gl

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cohort():
    return synth.make_cohort(40, 3000, 71, missing=0.02,
                             planted={"parent_offspring": 3, "full_sib": 3}, name="soft")


@pytest.fixture(scope="module")
def est():
    e = kb.Estimator()
    yield e
    e.close()


def test_soft_likelihoods_parity(est, oracle, cohort):
    gl = soft_gl(cohort.codes, np.random.default_rng(3), err=0.1)     # [sites, samples, 3]
    ref, _ = oracle.gl_relatedness(gl)
    est.load_likelihoods(np.ascontiguousarray(gl.transpose(1, 0, 2)))
    gpu = est.relatedness_gl()
    stats = compare(gpu, ref)
    same = float(np.mean(gpu["iters"] == ref["iters"]))
    print(stats, "same iterations", same)
    assert same > 0.95


def test_soft_subset_cap_and_maf(est, oracle, cohort):
    gl = soft_gl(cohort.codes, np.random.default_rng(4), err=0.05)
    ref, _ = oracle.gl_relatedness(gl, num_samples=25, iterations=5, maf=0.05)
    est.load_likelihoods(np.ascontiguousarray(gl.transpose(1, 0, 2)))
    gpu = est.relatedness_gl(num_samples=25, iterations=5, maf=0.05)
    assert gpu["iters"].max() <= 5
    assert np.mean(gpu["iters"] == ref["iters"]) > 0.95
    ok = ref["iters"] < 5
    d = np.abs(gpu["jacquard"] - ref["jacquard"]).max(1)
    lc = np.log10(ref["cond"])
    assert d[ok & np.isfinite(lc) & (lc < 15)].max() <= 1e-5


def test_one_hot_likelihoods_match_the_hard_call_path(est, oracle, cohort):
    # maf off the 1/(2N) tie (see the oracle tests)
    gl = one_hot(cohort.codes)
    est.load_likelihoods(np.ascontiguousarray(gl.transpose(1, 0, 2)))
    soft = est.relatedness_gl(maf=0.01)
    hard = oracle.relatedness(cohort.codes, maf=0.01)
    compare(soft, hard)


def test_python_gl_api_routes_soft_input(oracle, cohort):
    gl = soft_gl(cohort.codes, np.random.default_rng(5), err=0.1)
    jac, kin, inb = kb.relatedness_coefficients_gl(gl)
    ref, _ = oracle.gl_relatedness(gl)
    x, y = ref["x"].astype(int), ref["y"].astype(int)
    lc = np.log10(ref["cond"])
    below = np.isfinite(lc) & (lc < 15)
    assert np.abs(jac[x, y] - ref["jacquard"]).max(1)[below].max() <= 1e-5


def test_soft_entry_point_argument_errors(est):
    """maf above 1 and num_samples = 0 are refused with their own messages."""
    est.load_likelihoods(np.full((3, 4, 3), 0.5))
    for ns, maf, msg in ((-1, 1.5, "within 0 to 1"), (0, float("nan"), "must be positive")):
        with pytest.raises(kb.KestrelError) as ei:
            est.relatedness_gl(num_samples=ns if ns >= 0 else None, maf=maf)
        assert ei.value.status == kb.KG_EINVAL and msg in str(ei.value), str(ei.value)


def test_soft_fp32_and_fp64_forms(est, oracle, cohort):
    """Both evaluation forms against the oracle: FP32 evaluations (the default,
    with FP64 re-evaluation of pairs that need it) and the plain FP64 form."""
    gl = soft_gl(cohort.codes, np.random.default_rng(6), err=0.08)
    ref, _ = oracle.gl_relatedness(gl)
    est.load_likelihoods(np.ascontiguousarray(gl.transpose(1, 0, 2)))
    out = {}
    for prec in ("fp32c", "fp64"):
        est.set_precision(prec)
        rows = est.relatedness_gl()
        st = est.run_stats()
        out[prec] = (compare(rows, ref), {k: st[k] for k in ("gh_passes", "fp64_passes", "fp64_pairs", "work_units")})
    est.set_precision("fp32c")
    print(out)
    assert out["fp64"][1]["fp64_passes"] == out["fp64"][1]["gh_passes"] > 0
    assert out["fp32c"][1]["fp64_passes"] < out["fp32c"][1]["gh_passes"]


def _soft_multi(g, al, rng, err=0.05):
    """Tri- and tetra-allelic genotype indices (255 = missing) -> soft
    likelihoods [samples, sites, G] per allele count (the called genotype 1,
    the others uniform in [0, err)), NaN where missing."""
    out = {}
    for a in (3, 4):
        sel = np.nonzero(al == a)[0]
        ng = a * (a + 1) // 2
        sub = g[:, sel]
        gl = rng.uniform(0.0, err, sub.shape + (ng,))
        for k in range(ng):
            gl[..., k] = np.where(sub == k, 1.0, gl[..., k])
        gl[sub == 255] = np.nan
        out[a] = gl
    return out


def test_soft_multiallelic_sites_parity(est, oracle, cohort):
    """Tri- and tetra-allelic sites with soft likelihoods (kg_load_likelihoods_
    multiallelic) against the oracle's GL/PL path on the same likelihoods:
    frequencies fitted over 2-4 alleles, maf cut, zero-frequency alleles
    dropped, rows built from the remaining genotypes."""
    rng = np.random.default_rng(12)
    gl = soft_gl(cohort.codes, rng, err=0.08)                       # [sites, samples, 3]
    g, al = synth.make_multiallelic(cohort.codes.shape[0], 300, 13, missing=0.02)
    m = _soft_multi(g, al, rng)
    ref, af = oracle.gl_relatedness(gl, gl3=np.ascontiguousarray(m[3].transpose(1, 0, 2)),
                                    gl4=np.ascontiguousarray(m[4].transpose(1, 0, 2)))
    nz = (af > 0).sum(1)
    for prec in ("fp32c", "fp64"):
        est.set_precision(prec)
        est.load_likelihoods(np.ascontiguousarray(gl.transpose(1, 0, 2)))
        est.load_likelihoods_multiallelic(m[3], 3)
        est.load_likelihoods_multiallelic(m[4], 4)
        rows = est.relatedness_gl()
        st = est.run_stats()
        print(prec, compare(rows, ref), st["sites_used"], st["fp64_pairs"])
        assert st["sites_used"] == [int(np.sum(nz == 2)), int(np.sum(nz == 3)), int(np.sum(nz == 4))]
    est.set_precision("fp32c")
    assert st["sites_used"][1] > 0 and st["sites_used"][2] > 0


def test_cli_soft_pl_with_multiallelic_records(oracle):
    """The CLI on a soft PL VCF with tri- and tetra-allelic records: every
    record's likelihoods go to the soft estimator (10^(-PL/10), as the
    reference's reader makes them), against the oracle on the same arrays."""
    import os
    import subprocess
    import tempfile
    from .test_gpu_workloads import _read_tsv, _tsv_values
    from .parity import check_values
    from .test_vcf import py_likelihoods, soft_pl_text
    rng = np.random.default_rng(21)
    co = synth.make_cohort(22, 1200, seed=49, missing=0.02, name="cli-soft-multi")
    text = soft_pl_text(co.codes, rng)
    g, al = synth.make_multiallelic(22, 150, 50, missing=0.02)
    pls = {3: [], 4: []}
    lines = []
    for v in range(g.shape[1]):
        a = int(al[v])
        ng = a * (a + 1) // 2
        calls, row = [], []
        for s in range(22):
            if g[s, v] == 255:
                calls.append(".")
                row.append([np.nan] * ng)
                continue
            pl = rng.integers(5, 41, ng)
            pl[int(g[s, v])] = 0
            calls.append(",".join(str(int(x)) for x in pl))
            row.append([10.0 ** (-float(x) / 10.0) for x in pl])
        pls[a].append(row)
        lines.append(f"2\t{v + 1}\t.\tA\t{'C,G' if a == 3 else 'C,G,T'}\t.\tPASS\t.\tPL\t" + "\t".join(calls))
    text += "\n".join(lines) + "\n"
    gl2 = py_likelihoods(text.split("\n2\t")[0] + "\n", "PL")          # [samples, sites, 3]
    gl3 = np.array(pls[3])                                                # [sites, samples, 6]
    gl4 = np.array(pls[4])
    ref, _ = oracle.gl_relatedness(np.ascontiguousarray(gl2.transpose(1, 0, 2)), gl3=gl3, gl4=gl4)
    cli = os.path.join(os.path.dirname(kb.__file__), "bin", "kestrel")
    with tempfile.TemporaryDirectory() as td:
        vcf = os.path.join(td, "in.vcf")
        tsv = os.path.join(td, "out.tsv")
        open(vcf, "w").write(text)
        r = subprocess.run([cli, vcf, tsv, "-f", "PL"], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        _, rows = _read_tsv(tsv)
    assert "estimating from the soft likelihoods" in r.stderr
    assert f"Found {len(pls[3])} tri-allelic sites" in r.stderr
    assert len(rows) == len(ref)
    print(check_values(*_tsv_values(rows), ref))
