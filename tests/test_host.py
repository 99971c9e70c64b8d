"""Host-side pieces that need no GPU: the CLI's VCF reader and its errors, the
reference arm of bench.py, and the loud failure of the product path when no
CUDA device is present."""
import ctypes
import json
import os
import subprocess
import sys
import tempfile

import numpy as np
import pytest
import torch

import kestrel_b200 as kb
from kestrel_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "kestrel_b200", "bin", "kestrel")

HEADER = ("##fileformat=VCFv4.2\n##FORMAT=<ID=GT,Number=1,Type=String,Description=\"Genotype\">\n"
          "#CHROM\tPOS\tID\tREF\tALT\tQUAL\tFILTER\tINFO\tFORMAT\tA\tB\tC\n")


def _cli(args):
    return subprocess.run([CLI] + args, capture_output=True, text=True, timeout=120)


@pytest.fixture(scope="module")
def built():
    _lib.lib()   # the library and the CLI are built by the package build
    assert os.path.exists(CLI)


def test_cli_counts_skipped_records(built):
    recs = ["1\t1\t.\tA\tC\t.\tPASS\tAF=0.3\tGT\t0/0\t0/1\t1/1",
            "1\t2\t.\tA\tC,G\t.\tPASS\tAF=0.3\tGT\t0/0\t0/1\t1/2",     # tri-allelic
            "1\t3\t.\tAT\tC\t.\tPASS\tAF=0.3\tGT\t0/0\t0/1\t1/1",      # not a SNP
            "1\t4\t.\tG\tT\t.\tPASS\tAF=0.5\tGT\t0|1\t./.\t1/1",
            "1\t5\t.\tC\tA\t.\tPASS\tAF=0.1\tGT:DP\t0/0:3\t0/1:4\t0/0:5"]
    with tempfile.TemporaryDirectory() as td:
        vcf = os.path.join(td, "x.vcf")
        with open(vcf, "w") as fh:
            fh.write(HEADER + "\n".join(recs) + "\n")
        r = _cli([vcf, os.path.join(td, "o.tsv"), "-f", "GT"])
        r_ml = _cli([vcf, os.path.join(td, "o.tsv"), "-f", "GT", "-e", "ml"])
    for out in (r, r_ml):
        assert "Parsed 5 total sites" in out.stderr
        assert "Skipped 1 sites that were not SNPs" in out.stderr
    # GT runs CLS by default, on the records every sample calls (as the
    # reference's GT reader keeps), the tri-allelic one included; ML keeps the
    # record with a missing call and the tri-allelic one (the GL/PL reader's
    # counts)
    assert "Skipped 1 sites with missing data" in r.stderr
    assert "Found 2 di-allelic sites" in r.stderr
    assert "Found 1 tri-allelic sites" in r.stderr and "Found 0 tetra-allelic sites" in r.stderr
    assert "Found 3 di-allelic sites" in r_ml.stderr and "missing data" not in r_ml.stderr
    assert "Found 1 tri-allelic sites" in r_ml.stderr
    if not torch.cuda.is_available():
        assert r.returncode != 0


def test_cli_rejects_bad_input(built):
    with tempfile.TemporaryDirectory() as td:
        vcf = os.path.join(td, "bad.vcf")
        with open(vcf, "w") as fh:
            fh.write(HEADER + "1\t1\t.\tA\tC\t.\tPASS\t.\tGT\t0/0\t0/7\t1/1\n")
        r = _cli([vcf, os.path.join(td, "o.tsv")])
        assert r.returncode != 0 and "is not a valid GT" in r.stderr
        r = _cli([vcf, os.path.join(td, "o.tsv"), "-f", "XX"])
        assert r.returncode != 0
        r = _cli([os.path.join(td, "missing.vcf"), os.path.join(td, "o.tsv")])
        assert r.returncode != 0
        r = _cli([])
        assert r.returncode != 0 and "Usage" in r.stderr


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the behaviour without a CUDA device")
def test_product_path_fails_loudly_without_a_device():
    with pytest.raises(kb.KestrelError):
        kb.Estimator()
    codes = np.zeros((4, 16), np.uint8)
    out = np.empty(10, kb.OUTPUT_DTYPE)
    n = ctypes.c_int64()
    st = _lib.lib().kg_relatedness_coefficients(codes.ctypes.data, 4, 16, 16, None, 0, 100,
                                                float("nan"), 4, out.ctypes.data, out.size,
                                                ctypes.byref(n))
    assert st != _lib.KG_OK


def test_bench_reference_arm_prints_one_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--samples", "24", "--sites", "1500", "--steps", "1", "--warmup", "1",
                        "--cpu-seconds", "0.5"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "pairs/s" and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
