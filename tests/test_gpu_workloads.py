"""GPU tests of the serving path, the inbred stress cohort and the CLI, through
the C ABI, against the FP64 oracle (the same bar as test_gpu_parity.py)."""
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

import kestrel_b200 as kb
from kestrel_b200 import synth

from .parity import check_values, compare

pytestmark = pytest.mark.gpu


def _bitwise_equal(a, b):
    return a.shape == b.shape and np.array_equal(a.view(np.uint8), b.view(np.uint8))


@pytest.fixture(scope="module")
def panel():
    return synth.make_cohort(80, 3000, seed=21, name="panel")


def test_serving_alone_equals_mix_and_oracle(panel, oracle):
    reqs = synth.config4_requests(panel, 6, seed=5, max_query=5)
    with kb.Estimator() as est:
        est.panel_load(panel.codes)
        alone = [est.wait(est.submit(r["codes"], r["site_mask"])) for r in reqs]
        ids = [est.submit(r["codes"], r["site_mask"]) for r in reqs]    # all in flight together
        mixed = [est.wait(i) for i in ids]
        stats = est.serving_stats()
    for a, b, r in zip(alone, mixed, reqs):
        assert len(a) == r["codes"].shape[0] * panel.codes.shape[0]
        assert _bitwise_equal(a, b)
    assert stats["requests"] == 2 * len(reqs)
    # oracle: panel frequencies; the query's masked-out sites are missing
    p, q, keep = oracle.site_frequencies(panel.codes)
    for r, rows in list(zip(reqs, alone))[:2]:
        qc = r["codes"].copy()
        qc[:, ~r["site_mask"]] = 3
        nq, npn = qc.shape[0], panel.codes.shape[0]
        combined = np.vstack([qc, panel.codes])
        pairs = np.array([(i, nq + j) for i in range(nq) for j in range(npn)])
        ref = oracle.relatedness_pairs(combined, p, q, keep, pairs)
        assert np.array_equal(rows["x"], pairs[:, 0]) and np.array_equal(rows["y"], pairs[:, 1] - nq)
        print(compare(rows, ref, check_xy=False))


def test_serving_request_keeps_its_iteration_limit(panel):
    reqs = synth.config4_requests(panel, 3, seed=9, max_query=3)
    with kb.Estimator() as est:
        est.panel_load(panel.codes)
        alone = est.wait(est.submit(reqs[0]["codes"], reqs[0]["site_mask"], iterations=2))
        ids = [est.submit(reqs[0]["codes"], reqs[0]["site_mask"], iterations=2)] + \
              [est.submit(r["codes"], r["site_mask"], iterations=100) for r in reqs[1:]]
        mixed = [est.wait(i) for i in ids]
    assert np.all(alone["iters"] <= 2)
    assert _bitwise_equal(alone, mixed[0])


def test_serving_cancel(panel):
    reqs = synth.config4_requests(panel, 2, seed=13, max_query=2)
    with kb.Estimator() as est:
        est.panel_load(panel.codes)
        rid = est.submit(reqs[0]["codes"], reqs[0]["site_mask"])
        est.cancel(rid)
        keep = est.submit(reqs[1]["codes"], reqs[1]["site_mask"])
        rows = est.wait(keep)
        assert len(rows) == reqs[1]["codes"].shape[0] * panel.codes.shape[0]
        with pytest.raises(kb.KestrelError):
            est.wait(rid)


def test_inbred_stress_vs_oracle(oracle):
    co = synth.make_cohort(64, 5000, seed=31, planted={"identical_inbred": 4}, inbred=16,
                           low_info_sites=500, name="inbred")
    ref = oracle.relatedness(co.codes)
    with kb.Estimator() as est:
        est.load(co.codes)
        gpu = est.relatedness()
        st = est.run_stats()
    out = compare(gpu, ref)
    print(out, st["fp64_pairs"])
    lc = np.log10(ref["cond"])
    assert np.any(~(lc <= 15)), "the stress cohort should hold flagged pairs"
    # identical inbred pairs: Delta1 dominant
    for x, y, rel, delta in co.planted:
        i = int(np.nonzero((gpu["x"] == x) & (gpu["y"] == y))[0][0])
        assert gpu["jacquard"][i][0] > 0.5


def _tsv_values(rows):
    """Delta (jacquard1..9), objective and the log10 condition column of TSV rows."""
    jac = np.array([[float(v) for v in r[3:12]] for r in rows])
    obj = np.array([float(r[13]) for r in rows])
    lc = np.array([float(r[14]) for r in rows])
    return jac, obj, lc


_RESOURCE = re.compile(r"^\[INFO \] Wall Time [0-9.]+(s|ms|\u00b5s|ns), User Time [0-9.]+(s|ms|\u00b5s|ns), "
                       r"Kernel Time [0-9.]+(s|ms|\u00b5s|ns), Peak Memory [0-9.]+ (KiB|MiB|GiB|TiB)$")


def _resource_lines(stderr):
    """The reference's resource checkpoint lines (src/util.rs:34-36) in a log."""
    lines = [ln for ln in stderr.splitlines() if "Wall Time" in ln]
    assert all(_RESOURCE.match(ln) for ln in lines), lines
    return lines


def _read_tsv(path):
    with open(path) as fh:
        head = fh.readline().rstrip("\n").split("\t")
        rows = [ln.rstrip("\n").split("\t") for ln in fh]
    return head, rows


def test_cli_gt_and_pl_match_oracle(oracle):
    co = synth.make_cohort(24, 2500, seed=41, planted={"parent_offspring": 2})
    cli = os.path.join(os.path.dirname(kb.__file__), "bin", "kestrel")
    ref = oracle.relatedness(co.codes, num_samples=20)
    outs = {}
    with tempfile.TemporaryDirectory() as td:
        for field in ("GT", "PL"):
            vcf = os.path.join(td, f"in_{field}.vcf")
            tsv = os.path.join(td, f"out_{field}.tsv")
            synth.write_vcf(vcf, co.codes, field=field)
            r = subprocess.run([cli, vcf, tsv, "-f", field, "-s", "20", "-e", "ml"], capture_output=True,
                               text=True, timeout=300)
            assert r.returncode == 0, r.stderr
            # the ML path checks the reference's resource tracker twice
            assert len(_resource_lines(r.stderr)) == 2, r.stderr
            with open(tsv) as fh:
                outs[field] = fh.read()
            head, rows = _read_tsv(tsv)
    assert outs["GT"] == outs["PL"]
    assert head[:3] == ["sample1", "sample2", "kinship"] and head[-3:] == ["iterations", "objective",
                                                                          "condition"]
    assert len(rows) == len(ref)
    jac, obj, lc = _tsv_values(rows)
    kin = np.array([float(r[2]) for r in rows])
    print(check_values(jac, obj, lc, ref))
    assert np.abs(kin - jac @ kb.KINSHIP_VECTOR).max() <= 1e-12
    assert [r[0] for r in rows[:2]] == ["S0", "S0"] and [r[1] for r in rows[:2]] == ["S0", "S1"]


@pytest.mark.parametrize("threads", [1, 2, 5])
def test_cli_output_rows_equal_api_results(threads):
    # 33,930 pairs: more rows than one 16,384-row block per thread, so the
    # writer runs rounds, the last with idle threads (at -t 2)
    co = synth.make_cohort(260, 400, seed=44, name="cli-rows")
    cli = os.path.join(os.path.dirname(kb.__file__), "bin", "kestrel")
    with kb.Estimator() as est:
        est.load(co.codes)
        api = est.relatedness()
    with tempfile.TemporaryDirectory() as td:
        vcf = os.path.join(td, "in.vcf")
        tsv = os.path.join(td, "out.tsv")
        synth.write_vcf(vcf, co.codes, field="GT")
        r = subprocess.run([cli, vcf, tsv, "-t", str(threads), "-e", "ml"], capture_output=True, text=True,
                           timeout=300)
        assert r.returncode == 0, r.stderr
        _, rows = _read_tsv(tsv)
    assert len(rows) == len(api) == 260 * 261 // 2
    xy = np.array([[int(r[0][1:]), int(r[1][1:])] for r in rows])
    assert np.array_equal(xy[:, 0], api["x"]) and np.array_equal(xy[:, 1], api["y"])
    # shortest round-trip text: parsing gives back the API's doubles exactly
    jac = np.array([[float(v) for v in r[3:12]] for r in rows])
    assert np.array_equal(jac, api["jacquard"])
    assert np.array_equal(np.array([int(r[12]) for r in rows]), api["iters"].astype(np.int64))
    assert np.array_equal(np.array([float(r[13]) for r in rows]), api["obj"])


def test_cli_cls_estimator_matches_oracle(oracle):
    co = synth.make_cohort(24, 2500, seed=43, missing=0.0, planted={"parent_offspring": 2})
    cli = os.path.join(os.path.dirname(kb.__file__), "bin", "kestrel")
    ref = oracle.cls_relatedness(co.codes, num_samples=20)
    with tempfile.TemporaryDirectory() as td:
        vcf = os.path.join(td, "in.vcf")
        tsv = os.path.join(td, "out.tsv")
        synth.write_vcf(vcf, co.codes, field="GT")
        r = subprocess.run([cli, vcf, tsv, "-f", "GT", "-e", "cls", "-s", "20"], capture_output=True,
                           text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        head, rows = _read_tsv(tsv)
        # CLS is the default for GT, as in the reference's CLI
        tsv2 = os.path.join(td, "out_default.tsv")
        r2 = subprocess.run([cli, vcf, tsv2, "-s", "20"], capture_output=True, text=True, timeout=300)
        assert r2.returncode == 0, r2.stderr
        assert open(tsv).read() == open(tsv2).read()
        assert "Skipped 0 sites with missing data" in r2.stderr
        assert len(_resource_lines(r2.stderr)) == 1, r2.stderr
    assert len(rows) == len(ref)
    print(check_values(*_tsv_values(rows), ref))


def test_autotune_and_launch_shape_leave_results_unchanged(oracle):
    co = synth.make_cohort(300, 4000, seed=51)
    with kb.Estimator() as est:
        est.load(co.codes)
        base = est.relatedness()
        slots, bps = est.autotune()
        shape = est.launch()
        # the candidates kg_autotune times (0 = the defaults)
        assert slots == 0 and bps in (0, 4, 3)
        assert shape["unit_entries"] in (0, 65536, 16384, 8192) and shape["slot_divisor"] in (5, 3, 8)
        tuned = est.relatedness()
        est.set_work_unit(0)
        est.set_launch(64, 2)      # few slots in flight: many more waves
        small = est.relatedness()
        assert est.run_stats()["slots"] == 64
        est.set_work_unit(4096)    # other partial-sum groups: within the bar
        units = est.relatedness()
    assert _bitwise_equal(base, small)
    if shape["unit_entries"] == 0:
        assert _bitwise_equal(base, tuned)
    compare(tuned, base)
    compare(units, base)

def test_cli_gt_default_drops_records_with_missing_calls(oracle):
    co = synth.make_cohort(24, 4000, seed=45, missing=0.002, name="cli-cls-miss")
    incomplete = int(np.any(co.codes == synth.MISSING, 0).sum())
    assert 0 < incomplete < co.codes.shape[1]
    cli = os.path.join(os.path.dirname(kb.__file__), "bin", "kestrel")
    ref = oracle.cls_relatedness(co.codes)
    with tempfile.TemporaryDirectory() as td:
        vcf = os.path.join(td, "in.vcf")
        tsv = os.path.join(td, "out.tsv")
        synth.write_vcf(vcf, co.codes, field="GT")
        r = subprocess.run([cli, vcf, tsv], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        _, rows = _read_tsv(tsv)
    assert f"Skipped {incomplete} sites with missing data" in r.stderr
    assert f"Found {co.codes.shape[1] - incomplete} di-allelic sites" in r.stderr
    assert len(rows) == len(ref)
    print(check_values(*_tsv_values(rows), ref))


def test_cli_gt_default_fits_tri_and_tetra_allelic_records(oracle):
    co = synth.make_cohort(24, 3000, seed=46, missing=0.0, name="cli-multi")
    g, al = synth.make_multiallelic(24, 400, 47)
    g[3, 5] = 255                                        # skipped: a missing call
    ref = oracle.cls_relatedness(co.codes, multi=(g, al, None))
    cli = os.path.join(os.path.dirname(kb.__file__), "bin", "kestrel")
    alts = {3: "C,G", 4: "C,G,T"}
    lines = []
    for v in range(g.shape[1]):
        calls = []
        for s in range(24):
            if g[s, v] == 255:
                calls.append("./.")
                continue
            j = 0
            while (j + 1) * (j + 2) // 2 <= g[s, v]:
                j += 1
            calls.append(f"{g[s, v] - j * (j + 1) // 2}/{j}")
        lines.append(f"2\t{v + 1}\t.\tA\t{alts[int(al[v])]}\t.\tPASS\t.\tGT\t" + "\t".join(calls))
    with tempfile.TemporaryDirectory() as td:
        vcf = os.path.join(td, "in.vcf")
        tsv = os.path.join(td, "out.tsv")
        synth.write_vcf(vcf, co.codes, field="GT")
        with open(vcf, "a") as fh:
            fh.write("\n".join(lines) + "\n")
        r = subprocess.run([cli, vcf, tsv], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        _, rows = _read_tsv(tsv)
    n_tri = int(np.sum(al == 3)) - int(al[5] == 3)
    assert f"Found {n_tri} tri-allelic sites" in r.stderr
    assert f"Found {int(np.sum(al == 4)) - int(al[5] == 4)} tetra-allelic sites" in r.stderr
    assert "Skipped 1 sites with missing data" in r.stderr
    assert len(rows) == len(ref)
    print(check_values(*_tsv_values(rows), ref))


def test_packed_load_equals_byte_load():
    co = synth.make_cohort(70, 3001, seed=52, missing=0.02, name="packed")   # ragged last words
    c2, ob = kb.pack_2bit(co.codes)
    with kb.Estimator() as est:
        est.load(co.codes)
        ml, gt = est.relatedness(), est.relatedness_gt()
        est.load_packed(c2, ob, co.codes.shape[1])
        ml2, gt2 = est.relatedness(), est.relatedness_gt()
    assert _bitwise_equal(ml, ml2) and _bitwise_equal(gt, gt2)


def test_cli_soft_pl_file_uses_the_soft_estimator(oracle):
    from .test_vcf import py_likelihoods, soft_pl_text
    co = synth.make_cohort(24, 1500, seed=48, missing=0.02, name="cli-soft")
    text = soft_pl_text(co.codes, np.random.default_rng(2))
    gl = py_likelihoods(text, "PL")                      # [samples, sites, 3]
    ref, _ = oracle.gl_relatedness(np.ascontiguousarray(gl.transpose(1, 0, 2)), num_samples=20)
    cli = os.path.join(os.path.dirname(kb.__file__), "bin", "kestrel")
    with tempfile.TemporaryDirectory() as td:
        vcf = os.path.join(td, "in.vcf")
        tsv = os.path.join(td, "out.tsv")
        open(vcf, "w").write(text)
        r = subprocess.run([cli, vcf, tsv, "-f", "PL", "-s", "20"], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        _, rows = _read_tsv(tsv)
    assert "estimating from the soft likelihoods" in r.stderr
    assert len(rows) == len(ref)
    print(check_values(*_tsv_values(rows), ref))
