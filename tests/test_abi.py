"""CPU checks of the C-ABI library: it loads, exports every symbol the header
declares, and fails cleanly (an error status, no crash) without a GPU."""
import ctypes
import os
import re

import pytest

from kestrel_b200 import _lib
from kestrel_b200 import build as kbuild

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "kestrel_gpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(kg_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def L():
    kbuild.build()
    return _lib.lib()


def test_header_and_exports_agree(L):
    decl = declared_functions()
    assert set(decl) == set(_lib.EXPORTS)
    for name in decl:
        assert hasattr(L, name), name


def test_version_string(L):
    assert b"sm_100a" in L.kg_version()


def test_create_reports_error_without_gpu(L):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    st = L.kg_create(ctypes.byref(h), 0, 0)
    assert st == _lib.KG_ECUDA and not h.value


def test_null_context_is_einval(L):
    assert L.kg_set_precision(None, 0) == _lib.KG_EINVAL
    assert L.kg_relatedness(None, -1, 100, 0.0, None, 0, None) == _lib.KG_EINVAL
    assert L.kg_destroy(None) == _lib.KG_EINVAL


def test_cli_usage_error_without_gpu(L):
    argv = (ctypes.c_char_p * 2)(b"kestrel", b"--bogus")
    assert L.kg_run_cli(2, argv) == 2


def test_cli_cls_needs_hard_calls(L):
    argv = (ctypes.c_char_p * 7)(b"kestrel", b"in.vcf", b"out.tsv", b"-f", b"PL", b"-e", b"cls")
    assert L.kg_run_cli(7, argv) == 2


def test_soft_likelihood_entry_points_check_their_arguments(L):
    # argument checks only: no device work (kg_create is not called)
    assert L.kg_load_likelihoods(None, None, 1, 1) == _lib.KG_EINVAL
    assert L.kg_relatedness_gl(None, -1, 100, float("nan"), None, 0, None) == _lib.KG_EINVAL
    assert L.kg_vcf_likelihoods(None, None) == _lib.KG_EINVAL

