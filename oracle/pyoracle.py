"""ctypes binding of the FP64 oracle — TEST INFRASTRUCTURE ONLY.

Only tests, the smoke check and the benchmark's CPU-baseline leg import this
module.  The oracle is a restatement of the reference's ML Jacquard estimator;
its parity with the reference is unpinned (see kestrel_oracle.h).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libkestrel_oracle.so")


class KorOutput(ctypes.Structure):
    _fields_ = [("x", ctypes.c_uint64), ("y", ctypes.c_uint64),
                ("jacquard", ctypes.c_double * 9), ("obj", ctypes.c_double),
                ("iters", ctypes.c_uint64), ("cond", ctypes.c_double)]


OUTPUT_DTYPE = np.dtype([("x", np.uint64), ("y", np.uint64), ("jacquard", np.float64, 9),
                         ("obj", np.float64), ("iters", np.uint64), ("cond", np.float64)])
assert OUTPUT_DTYPE.itemsize == ctypes.sizeof(KorOutput)

_lib = None


def build() -> str:
    """Compiles the oracle library in place (make)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        i64, u64, dbl = ctypes.c_int64, ctypes.c_uint64, ctypes.c_double
        P = ctypes.c_void_p
        L.kor_site_frequencies.argtypes = [P, i64, i64, i64, P, dbl, P, P, P, ctypes.POINTER(i64)]
        L.kor_site_frequencies_it.argtypes = [P, i64, i64, i64, P, dbl, u64, P, P, P, ctypes.POINTER(i64)]
        L.kor_relatedness.argtypes = [P, i64, i64, i64, P, i64, u64, dbl, ctypes.c_int, P, i64,
                                      ctypes.POINTER(i64)]
        L.kor_relatedness_pairs.argtypes = [P, i64, i64, P, P, P, P, P, i64, u64, ctypes.c_int, P]
        L.kor_eval_pair.argtypes = [P, P, i64, P, P, P, P, P, P, P, ctypes.POINTER(i64)]
        L.kor_allele_counts.argtypes = [P, i64, i64, i64, P, P]
        L.kor_pass_counts.argtypes = [ctypes.POINTER(u64), ctypes.POINTER(u64)]
        L.kor_cls_relatedness.argtypes = [P, i64, i64, i64, P, i64, u64, ctypes.c_int, P, i64,
                                          ctypes.POINTER(i64)]
        L.kor_cls_relatedness_ma.argtypes = [P, i64, i64, i64, P, P, i64, i64, P, P, i64, u64,
                                             ctypes.c_int, P, i64, ctypes.POINTER(i64)]
        L.kor_iis_row.argtypes = [ctypes.c_int, ctypes.c_int, P, P]
        L.kor_gl_relatedness.argtypes = [P, i64, P, i64, P, i64, i64, dbl, i64, u64, ctypes.c_int, P, i64,
                                         ctypes.POINTER(i64), P]
        L.kor_gl_allele_frequencies.argtypes = [P, i64, i64, ctypes.c_int, u64, dbl, ctypes.c_int, P]
        L.kor_iis_row.restype = None
        for f in ("kor_site_frequencies", "kor_site_frequencies_it", "kor_relatedness", "kor_relatedness_pairs",
                  "kor_eval_pair", "kor_allele_counts", "kor_cls_relatedness", "kor_cls_relatedness_ma",
                  "kor_gl_relatedness", "kor_gl_allele_frequencies"):
            getattr(L, f).restype = ctypes.c_int
        L.kor_pass_counts.restype = None
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def _codes(codes):
    codes = np.ascontiguousarray(codes, dtype=np.uint8)
    assert codes.ndim == 2
    return codes


def allele_counts(codes):
    codes = _codes(codes)
    n, m = codes.shape
    rc = np.zeros(m, np.int32)
    oc = np.zeros(m, np.int32)
    st = lib().kor_allele_counts(_ptr(codes), n, m, m, _ptr(rc), _ptr(oc))
    if st:
        raise RuntimeError(f"kor_allele_counts failed: {st}")
    return rc, oc


def site_frequencies(codes, af=None, maf=None, iterations=100):
    codes = _codes(codes)
    n, m = codes.shape
    p = np.zeros(m)
    q = np.zeros(m)
    keep = np.zeros(m, np.uint8)
    kept = ctypes.c_int64()
    afa = None if af is None else np.ascontiguousarray(af, dtype=np.float64)
    st = lib().kor_site_frequencies_it(_ptr(codes), n, m, m, _ptr(afa),
                                       -1.0 if maf is None else float(maf), iterations,
                                       _ptr(p), _ptr(q), _ptr(keep), ctypes.byref(kept))
    if st:
        raise RuntimeError(f"kor_site_frequencies failed: {st}")
    return p, q, keep.astype(bool)


def relatedness(codes, af=None, num_samples=None, iterations=100, maf=None, threads=0):
    codes = _codes(codes)
    n, m = codes.shape
    ns = n if num_samples is None else num_samples
    out = np.zeros(ns * (ns + 1) // 2, OUTPUT_DTYPE)
    nout = ctypes.c_int64()
    afa = None if af is None else np.ascontiguousarray(af, dtype=np.float64)
    st = lib().kor_relatedness(_ptr(codes), n, m, m, _ptr(afa), ns, iterations,
                               -1.0 if maf is None else float(maf), threads,
                               _ptr(out), out.size, ctypes.byref(nout))
    if st:
        raise RuntimeError(f"kor_relatedness failed: {st}")
    return out


def cls_relatedness(codes, af=None, num_samples=None, iterations=100, threads=0, multi=None):
    """The reference's default hard-call estimator (conditional least squares,
    Brier objective): rows as `relatedness`, obj = Brier score, iters = QP
    iterations.  multi: None or (genotype indices u8 [samples, sites] in the VCF
    order with 255 = missing, allele counts u8 [sites] of 3 or 4, allele
    frequencies f64 [sites, 4] or None) for tri- and tetra-allelic sites."""
    codes = _codes(codes)
    n, m = codes.shape
    ns = n if num_samples is None else num_samples
    out = np.zeros(ns * (ns + 1) // 2, OUTPUT_DTYPE)
    nout = ctypes.c_int64()
    afa = None if af is None else np.ascontiguousarray(af, dtype=np.float64)
    if multi is None:
        st = lib().kor_cls_relatedness(_ptr(codes), n, m, m, _ptr(afa), ns, iterations, threads,
                                       _ptr(out), out.size, ctypes.byref(nout))
    else:
        mg = np.ascontiguousarray(multi[0], dtype=np.uint8)
        mal = np.ascontiguousarray(multi[1], dtype=np.uint8)
        maf = None if len(multi) < 3 or multi[2] is None else np.ascontiguousarray(multi[2], dtype=np.float64)
        assert mg.shape[0] == n and mg.shape[1] == mal.shape[0]
        vm = mg.shape[1]
        st = lib().kor_cls_relatedness_ma(_ptr(codes), n, m, m, _ptr(afa), _ptr(mg), vm, vm, _ptr(mal),
                                          _ptr(maf), ns, iterations, threads, _ptr(out), out.size,
                                          ctypes.byref(nout))
    if st:
        raise RuntimeError(f"kor_cls_relatedness failed: {st}")
    return out


def iis_row(gx, gy, freq):
    """m[gx][gy] (9 conditional probabilities) for genotype indices in the VCF
    order and allele frequencies freq."""
    f = np.zeros(4)
    f[:len(freq)] = freq
    row = np.zeros(9)
    lib().kor_iis_row(int(gx), int(gy), _ptr(f), _ptr(row))
    return row


def relatedness_pairs(codes, p, q, keep, pairs, iterations=100, threads=0):
    codes = _codes(codes)
    n, m = codes.shape
    pairs = np.asarray(pairs, dtype=np.int64).reshape(-1, 2)
    px = np.ascontiguousarray(pairs[:, 0])
    py = np.ascontiguousarray(pairs[:, 1])
    out = np.zeros(len(pairs), OUTPUT_DTYPE)
    keep8 = np.ascontiguousarray(keep, dtype=np.uint8)
    p = np.ascontiguousarray(p, dtype=np.float64)
    q = np.ascontiguousarray(q, dtype=np.float64)
    st = lib().kor_relatedness_pairs(_ptr(codes), m, m, _ptr(p), _ptr(q), _ptr(keep8),
                                     _ptr(px), _ptr(py), len(pairs), iterations, threads,
                                     _ptr(out))
    if st:
        raise RuntimeError(f"kor_relatedness_pairs failed: {st}")
    return out


def pass_counts():
    gh = ctypes.c_uint64()
    ob = ctypes.c_uint64()
    lib().kor_pass_counts(ctypes.byref(gh), ctypes.byref(ob))
    return gh.value, ob.value


def eval_pair(codes_x, codes_y, p, q, keep, delta):
    cx = np.ascontiguousarray(codes_x, dtype=np.uint8)
    cy = np.ascontiguousarray(codes_y, dtype=np.uint8)
    keep8 = np.ascontiguousarray(keep, dtype=np.uint8)
    p = np.ascontiguousarray(p, dtype=np.float64)
    q = np.ascontiguousarray(q, dtype=np.float64)
    d = np.ascontiguousarray(delta, dtype=np.float64)
    f = ctypes.c_double()
    g = np.zeros(9)
    h = np.zeros(81)
    n = ctypes.c_int64()
    st = lib().kor_eval_pair(_ptr(cx), _ptr(cy), cx.size, _ptr(p), _ptr(q), _ptr(keep8),
                             _ptr(d), ctypes.byref(f), _ptr(g), _ptr(h), ctypes.byref(n))
    if st:
        raise RuntimeError(f"kor_eval_pair failed: {st}")
    return f.value, g, h.reshape(9, 9), n.value


def gl_relatedness(gl2, gl3=None, gl4=None, maf=None, num_samples=None, iterations=100, threads=0):
    """The GL/PL estimator on soft likelihoods: gl2 [sites, samples, 3], gl3
    [sites, samples, 6], gl4 [sites, samples, 10], linear scale, NaN = missing.
    Returns (rows, allele frequencies [sites, 4] in input order)."""
    arrs = []
    n = None
    for a, g in ((gl2, 3), (gl3, 6), (gl4, 10)):
        if a is None:
            arrs.append(None)
            continue
        a = np.ascontiguousarray(a, dtype=np.float64)
        assert a.ndim == 3 and a.shape[2] == g
        n = a.shape[1] if n is None else n
        assert a.shape[1] == n
        arrs.append(a)
    counts = [0 if a is None else a.shape[0] for a in arrs]
    ns = n if num_samples is None else num_samples
    out = np.zeros(ns * (ns + 1) // 2, OUTPUT_DTYPE)
    af = np.zeros((sum(counts), 4))
    nout = ctypes.c_int64()
    st = lib().kor_gl_relatedness(_ptr(arrs[0]), counts[0], _ptr(arrs[1]), counts[1], _ptr(arrs[2]), counts[2], n,
                                  float("nan") if maf is None else float(maf), ns, iterations, threads, _ptr(out),
                                  out.size, ctypes.byref(nout), _ptr(af))
    if st:
        raise RuntimeError(f"kor_gl_relatedness failed: {st}")
    return out, af


def gl_allele_frequencies(gl, maf=0.0, iterations=100, threads=0):
    """Per-site allele frequencies from likelihoods [sites, samples, G]."""
    gl = np.ascontiguousarray(gl, dtype=np.float64)
    g = gl.shape[2]
    a = {3: 2, 6: 3, 10: 4}[g]
    af = np.zeros((gl.shape[0], 4))
    st = lib().kor_gl_allele_frequencies(_ptr(gl), gl.shape[0], gl.shape[1], a, iterations, float(maf), threads,
                                         _ptr(af))
    if st:
        raise RuntimeError(f"kor_gl_allele_frequencies failed: {st}")
    return af
