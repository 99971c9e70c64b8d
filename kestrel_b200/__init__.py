"""kestrel_b200 — B200-native all-pairs maximum-likelihood Jacquard estimator.

Python surface of the reference's `kestrel` module (src/lib.rs:26-161):
`relatedness_coefficients_gt`, `relatedness_coefficients_gl`, `run_cli` and
`Coefficients`, all running on libkestrel_gpu.so (sm_100a).  `Estimator` exposes
the context API (precision, batching of several cohorts, serving a resident
panel) of include/kestrel_gpu.h.
"""
from __future__ import annotations

import ctypes
import os
import sys
import warnings

import numpy as np

from ._lib import (KG_ECUDA, KG_EINVAL, KG_ENOMEM, KG_ENOSITES, KG_ENOTFOUND, KG_ENOTREADY, KG_ETIMEOUT, KG_OK,
                   KG_PREC_FP32C, KG_PREC_FP64, MISSING, OUTPUT_DTYPE, KestrelError, KgCohort, KgRunStats, lib,
                   ptr)

__all__ = ["Coefficients", "relatedness_coefficients_gt", "relatedness_coefficients_gl", "read_vcf", "pack_2bit",
           "read_vcf_likelihoods",
           "run_cli", "Estimator", "genotype_codes", "build_arrays", "KestrelError",
           "OUTPUT_DTYPE", "MISSING", "KINSHIP_VECTOR", "KG_OK", "KG_EINVAL", "KG_ENOMEM", "KG_ECUDA",
           "KG_ETIMEOUT", "KG_ENOSITES", "KG_ENOTREADY", "KG_ENOTFOUND", "KG_PREC_FP32C", "KG_PREC_FP64"]

# Kinship as a linear function of Delta (src/cli.rs:150, src/lib.rs:127).
KINSHIP_VECTOR = np.array([1.0, 0.0, 0.5, 0.0, 0.5, 0.0, 0.5, 0.25, 0.0])


class Coefficients:
    """Result arrays of the reference's Python API (src/lib.rs:36-44)."""

    def __init__(self, jacquard, kinship, inbreeding):
        self.jacquard = jacquard
        self.kinship = kinship
        self.inbreeding = inbreeding

    def __repr__(self):
        return f"Coefficients(samples={self.kinship.shape[0]})"


def _check(status: int, ctx=None):
    if status != KG_OK:
        msg = lib().kg_last_error(ctx).decode() if ctx else ""
        raise KestrelError(status, msg)


def genotype_codes(genotypes: np.ndarray) -> np.ndarray:
    """u8/int [V, S, 2] allele indices -> sample-major [S, V] codes 0/1/2, 3 = missing.

    The unphased index j(j+1)/2 + i of the reference (src/coefficients.rs:19-38)
    for biallelic sites; an allele < 0 or > 1 (e.g. -1 or 255) marks a missing call.
    """
    g = np.asarray(genotypes)
    if g.ndim != 3 or g.shape[2] != 2:
        raise ValueError("genotypes must have shape (variants, samples, 2)")
    a = g.astype(np.int16)
    if g.dtype == np.uint8:
        a = np.where(g == 255, -1, a)
    miss = (a < 0) | (a > 1)
    codes = (a[..., 0] + a[..., 1]).astype(np.uint8)
    codes[miss.any(axis=2)] = MISSING
    return np.ascontiguousarray(codes.T)


def pack_2bit(codes: np.ndarray):
    """Sample-major codes [samples, sites] (3 = missing) -> the packed form of
    kg_load_genotypes_2bit: (2-bit codes uint32 [samples, ceil(sites/16)], site
    s at bits 2 (s % 16), 0 where missing; observed mask uint32 [samples,
    ceil(sites/32)], bit s % 32)."""
    c = np.ascontiguousarray(codes, dtype=np.uint8)
    n, m = c.shape
    called = c < 3
    m16, m32 = -(-m // 16) * 16, -(-m // 32) * 32
    cc = np.zeros((n, m16), np.uint32)
    cc[:, :m] = np.where(called, c, 0)
    codes2 = (cc.reshape(n, -1, 16) << (2 * np.arange(16, dtype=np.uint32))).sum(2, dtype=np.uint64).astype(np.uint32)
    ob = np.zeros((n, m32), np.uint32)
    ob[:, :m] = called
    observed = (ob.reshape(n, -1, 32) << np.arange(32, dtype=np.uint32)).sum(2, dtype=np.uint64).astype(np.uint32)
    return np.ascontiguousarray(codes2), np.ascontiguousarray(observed)


def build_arrays(rows: np.ndarray, num_samples: int):
    """(jacquard N x N x 9, kinship N x N, inbreeding N) from output rows, with
    the D3<->D5 and D4<->D6 swap for (y, x) (src/lib.rs:120-161)."""
    jac = np.zeros((num_samples, num_samples, 9))
    kin = np.zeros((num_samples, num_samples))
    inb = np.zeros(num_samples)
    x = rows["x"].astype(np.int64)
    y = rows["y"].astype(np.int64)
    d = rows["jacquard"]
    k = d @ KINSHIP_VECTOR
    jac[x, y] = d
    off = x != y
    jac[y[off], x[off]] = d[off][:, [0, 1, 4, 5, 2, 3, 6, 7, 8]]
    kin[x, y] = k
    kin[y[off], x[off]] = k[off]
    self_ = ~off
    inb[x[self_]] = 2.0 * k[self_] - 1.0
    return jac, kin, inb


class Estimator:
    """A device context (kg_ctx) on one GPU."""

    def __init__(self, device: int = 0, mem_budget: int = 0, precision: str = "fp32c"):
        self._L = lib()
        h = ctypes.c_void_p()
        st = self._L.kg_create(ctypes.byref(h), device, mem_budget)
        if st != KG_OK:
            raise KestrelError(st, "kg_create failed (is a CUDA device present?)")
        self._h = h
        self.n_samples = 0
        self.n_sites = 0
        self.set_precision(precision)

    def close(self):
        if getattr(self, "_h", None):
            self._L.kg_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_precision(self, precision: str):
        p = {"fp32c": KG_PREC_FP32C, "fp64": KG_PREC_FP64}[precision]
        _check(self._L.kg_set_precision(self._h, p), self._h)

    def set_launch(self, slots: int = 0, blocks_per_sm: int = 0):
        """Pairs in flight per wave and site-pass blocks per SM (0 = automatic)."""
        _check(self._L.kg_set_launch(self._h, slots, blocks_per_sm), self._h)

    def set_wave_limit(self, waves: int = 0):
        """Waves a call may run before it stops with KG_ETIMEOUT (0 = a bound
        from the work, which only stops a loop that would not end)."""
        _check(self._L.kg_set_wave_limit(self._h, int(waves)), self._h)

    def set_work_unit(self, entries: int = 0):
        """List entries per site-pass work unit (0 = the default, 32768)."""
        _check(self._L.kg_set_work_unit(self._h, int(entries)), self._h)

    def launch(self) -> dict:
        """The launch shape in use (kg_get_launch; 0 = automatic / default)."""
        v = [ctypes.c_int() for _ in range(4)]
        _check(self._L.kg_get_launch(self._h, *[ctypes.byref(x) for x in v]), self._h)
        return dict(zip(("slots", "blocks_per_sm", "unit_entries", "slot_divisor"), (x.value for x in v)))

    def autotune(self):
        """Runs kg_autotune; returns (slots, blocks_per_sm) as the C call does
        (launch() gives the work unit and the slot divisor it chose)."""
        w, b = ctypes.c_int(), ctypes.c_int()
        _check(self._L.kg_autotune(self._h, ctypes.byref(w), ctypes.byref(b)), self._h)
        return w.value, b.value

    def load(self, codes: np.ndarray, allele_frequencies=None):
        codes = np.ascontiguousarray(codes, dtype=np.uint8)
        if codes.ndim != 2:
            raise ValueError("codes must be (samples, sites)")
        n, m = codes.shape
        _check(self._L.kg_load_genotypes(self._h, ptr(codes), n, m, m), self._h)
        self.n_samples, self.n_sites = n, m
        if allele_frequencies is not None:
            af = np.ascontiguousarray(allele_frequencies, dtype=np.float64)
            if af.shape != (m, 2):
                raise ValueError("allele_frequencies must be (sites, 2)")
            _check(self._L.kg_set_allele_frequencies(self._h, ptr(af)), self._h)
            self._af = af
        return self

    def load_packed(self, codes2: np.ndarray, observed: np.ndarray, n_sites: int, allele_frequencies=None):
        """Loads a cohort from the packed form (pack_2bit, the VCF reader's
        read_vcf(..., packed=True)): unpacked to byte codes on the device."""
        c2 = np.ascontiguousarray(codes2, dtype=np.uint32)
        ob = np.ascontiguousarray(observed, dtype=np.uint32)
        n = c2.shape[0]
        if c2.shape != (n, -(-n_sites // 16)) or ob.shape != (n, -(-n_sites // 32)):
            raise ValueError("codes2 must be (samples, ceil(sites/16)) and observed (samples, ceil(sites/32))")
        _check(self._L.kg_load_genotypes_2bit(self._h, ptr(c2), ptr(ob), n, int(n_sites)), self._h)
        self.n_samples, self.n_sites = n, int(n_sites)
        if allele_frequencies is not None:
            af = np.ascontiguousarray(allele_frequencies, dtype=np.float64)
            if af.shape != (n_sites, 2):
                raise ValueError("allele_frequencies must be (sites, 2)")
            _check(self._L.kg_set_allele_frequencies(self._h, ptr(af)), self._h)
            self._af = af
        return self

    def load_likelihoods(self, likelihoods: np.ndarray):
        """Soft genotype likelihoods for relatedness_gl: double [samples, sites,
        3] (0/0, 0/1, 1/1), linear scale, NaN = missing."""
        gl = np.ascontiguousarray(likelihoods, dtype=np.float64)
        if gl.ndim != 3 or gl.shape[2] != 3:
            raise ValueError("likelihoods must be (samples, sites, 3)")
        _check(self._L.kg_load_likelihoods(self._h, ptr(gl), gl.shape[0], gl.shape[1]), self._h)
        self.n_gl_samples = gl.shape[0]
        return self

    def load_likelihoods_multiallelic(self, likelihoods: np.ndarray, n_alleles: int):
        """Tri- (G = 6) or tetra-allelic (G = 10) sites for relatedness_gl:
        double [samples, sites, G], genotypes in the VCF order, linear scale,
        NaN = missing; after load_likelihoods."""
        gl = np.ascontiguousarray(likelihoods, dtype=np.float64)
        ng = n_alleles * (n_alleles + 1) // 2
        if gl.ndim != 3 or gl.shape[2] != ng:
            raise ValueError(f"likelihoods must be (samples, sites, {ng})")
        _check(self._L.kg_load_likelihoods_multiallelic(self._h, ptr(gl), gl.shape[0], gl.shape[1], int(n_alleles)),
               self._h)
        return self

    def relatedness_gl(self, num_samples=None, iterations: int = 100, maf=None,
                       out: np.ndarray | None = None) -> np.ndarray:
        """The GL/PL estimator on the loaded soft likelihoods (kg_relatedness_gl)."""
        ns = getattr(self, "n_gl_samples", 0) if num_samples is None else int(num_samples)
        np_ = ns * (ns + 1) // 2
        if out is None:
            out = np.empty(np_, OUTPUT_DTYPE)
        nout = ctypes.c_int64()
        _check(self._L.kg_relatedness_gl(self._h, ns, iterations, float("nan") if maf is None else float(maf),
                                         ptr(out), out.size, ctypes.byref(nout)), self._h)
        return out

    def load_multiallelic(self, genotype_indices: np.ndarray, n_alleles, allele_frequencies=None):
        """Tri- and tetra-allelic sites for relatedness_gt: genotype indices u8
        [samples, sites] in the VCF order (j (j + 1) / 2 + i, 255 = missing),
        allele counts [sites] (3 or 4), frequencies [sites, 4] or None."""
        g = np.ascontiguousarray(genotype_indices, dtype=np.uint8)
        if g.ndim != 2 or g.shape[0] != self.n_samples:
            raise ValueError("genotype_indices must be (samples, sites) with the loaded samples")
        na = np.ascontiguousarray(n_alleles, dtype=np.uint8)
        if na.shape != (g.shape[1],):
            raise ValueError("n_alleles must have one entry per site")
        af = None
        if allele_frequencies is not None:
            af = np.ascontiguousarray(allele_frequencies, dtype=np.float64)
            if af.shape != (g.shape[1], 4):
                raise ValueError("allele_frequencies must be (sites, 4)")
        _check(self._L.kg_load_multiallelic(self._h, ptr(g), g.shape[0], g.shape[1], g.shape[1], ptr(na), ptr(af)),
               self._h)
        self._multi = (g, na, af)
        return self

    def relatedness(self, num_samples=None, iterations: int = 100, maf=None,
                    out: np.ndarray | None = None, allow_nosites: bool = False) -> np.ndarray:
        ns = self.n_samples if num_samples is None else int(num_samples)
        np_ = ns * (ns + 1) // 2
        if out is None:
            out = np.empty(np_, OUTPUT_DTYPE)
        nout = ctypes.c_int64()
        st = self._L.kg_relatedness(self._h, ns, iterations,
                                    float("nan") if maf is None else float(maf),
                                    ptr(out), out.size, ctypes.byref(nout))
        if st == KG_ENOSITES and allow_nosites and nout.value == np_:
            return out
        _check(st, self._h)
        return out

    def relatedness_gt(self, num_samples=None, iterations: int = 100,
                       out: np.ndarray | None = None) -> np.ndarray:
        """The reference's default hard-call estimator (-f GT): conditional least
        squares with the Brier objective (calculate_relatedness_coefficients_gt).
        Rows as `relatedness`; obj is the Brier score and iters the QP
        iterations.  Only sites every loaded sample calls are used."""
        ns = self.n_samples if num_samples is None else int(num_samples)
        np_ = ns * (ns + 1) // 2
        if out is None:
            out = np.empty(np_, OUTPUT_DTYPE)
        nout = ctypes.c_int64()
        st = self._L.kg_relatedness_gt(self._h, ns, iterations, ptr(out), out.size, ctypes.byref(nout))
        _check(st, self._h)
        return out

    def run_stats(self) -> dict:
        s = KgRunStats()
        _check(self._L.kg_last_run_stats(self._h, ctypes.byref(s)), self._h)
        d = {f: getattr(s, f) for f, _ in KgRunStats._fields_}
        d["shape_sites"] = list(s.shape_sites)
        d["sites_used"] = list(s.sites_used)
        return d

    def relatedness_batch(self, cohorts, iterations: int = 100, maf=None, out=None):
        """cohorts: list of (codes[S, V] u8, allele_frequencies or None, num_samples or None).
        Returns one row array per cohort, all from a single persistent launch.
        out: optional list of row arrays (OUTPUT_DTYPE, at least num_samples *
        (num_samples + 1) / 2 rows each), filled and returned in place (page-locked
        ones avoid first-touch page faults in the copy back)."""
        arr = (KgCohort * len(cohorts))()
        keep = []
        outs = []
        for i, c in enumerate(cohorts):
            codes, af, ns = (list(c) + [None, None])[:3]
            codes = np.ascontiguousarray(codes, dtype=np.uint8)
            n, m = codes.shape
            ns = n if ns is None else int(ns)
            if out is not None:
                o = out[i]
                if o.dtype != OUTPUT_DTYPE or o.ndim != 1 or o.size < ns * (ns + 1) // 2:
                    raise ValueError(f"out[{i}] must be a 1-D {OUTPUT_DTYPE} array of at least "
                                     f"{ns * (ns + 1) // 2} rows")
                out_i = o
            else:
                out_i = np.empty(ns * (ns + 1) // 2, OUTPUT_DTYPE)
            afa = None if af is None else np.ascontiguousarray(af, dtype=np.float64)
            keep += [codes, afa, out_i]
            arr[i].codes = codes.ctypes.data
            arr[i].n_samples, arr[i].n_sites, arr[i].row_stride = n, m, m
            arr[i].allele_frequencies = None if afa is None else afa.ctypes.data
            arr[i].num_samples = ns
            arr[i].out = out_i.ctypes.data
            arr[i].out_cap = out_i.size
            outs.append(out_i)
        st = self._L.kg_relatedness_batch(self._h, arr, len(cohorts), iterations,
                                          float("nan") if maf is None else float(maf))
        _check(st, self._h)
        return outs

    # ---- serving
    def panel_load(self, codes: np.ndarray, allele_frequencies=None, maf=None):
        codes = np.ascontiguousarray(codes, dtype=np.uint8)
        n, m = codes.shape
        afa = None if allele_frequencies is None else np.ascontiguousarray(allele_frequencies, np.float64)
        _check(self._L.kg_panel_load(self._h, ptr(codes), n, m, m, ptr(afa),
                                     float("nan") if maf is None else float(maf)), self._h)
        self.panel_samples, self.panel_sites = n, m

    def submit(self, query_codes: np.ndarray, site_mask=None, iterations: int = 100) -> int:
        q = np.ascontiguousarray(query_codes, dtype=np.uint8)
        mask = None if site_mask is None else np.ascontiguousarray(site_mask, dtype=np.uint8)
        rid = ctypes.c_int64()
        _check(self._L.kg_submit(self._h, ptr(q), q.shape[0], q.shape[1], ptr(mask), iterations,
                                 ctypes.byref(rid)), self._h)
        self._pending = getattr(self, "_pending", {})
        self._pending[rid.value] = q.shape[0]
        return rid.value

    def poll(self, request_id: int) -> bool:
        done = ctypes.c_int()
        _check(self._L.kg_poll(self._h, request_id, ctypes.byref(done)), self._h)
        return bool(done.value)

    def wait(self, request_id: int, timeout_ms: int = -1) -> np.ndarray | None:
        nq = self._pending.get(request_id, 0)
        out = np.empty(max(nq * self.panel_samples, 1), OUTPUT_DTYPE)
        nout = ctypes.c_int64()
        st = self._L.kg_wait(self._h, request_id, timeout_ms, ptr(out), out.size, ctypes.byref(nout))
        if st == KG_ETIMEOUT:
            return None
        self._pending.pop(request_id, None)
        _check(st, self._h)
        return out[:nout.value]

    def cancel(self, request_id: int):
        _check(self._L.kg_cancel(self._h, request_id), self._h)

    def serving_stats(self):
        r, p, l_ = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        _check(self._L.kg_serving_stats(self._h, ctypes.byref(r), ctypes.byref(p), ctypes.byref(l_)),
               self._h)
        return {"requests": r.value, "pairs": p.value, "launches": l_.value}


def relatedness_coefficients_gt(genotypes, allele_frequencies=None, threads=None, iterations=100,
                                estimator="ml"):
    """Jacquard, kinship and inbreeding for every pair of samples from hard
    calls (the reference's signature, src/lib.rs:46-70).  genotypes: u8/int
    [variants, samples, 2] allele indices; allele_frequencies: f64 [variants, 2]
    ([REF, ALT]) or None to estimate.  `threads` is accepted and unused.
    Sites whose calls use allele 2 or 3 are tri- or tetra-allelic (their
    allele count is the largest allele + 1); allele_frequencies, when given,
    are [variants, 2] for the biallelic sites only.  estimator "ml" runs the
    maximum-likelihood estimator on the calls (the reference's GL/PL path on
    one-hot likelihoods); "cls" runs the reference's own hard-call estimator
    (conditional least squares with the Brier objective,
    src/coefficients.rs:166-278) on the sites every sample calls."""
    del threads
    if estimator not in ("ml", "cls"):
        raise ValueError("estimator must be 'ml' or 'cls'")
    g = np.asarray(genotypes)
    if g.ndim != 3 or g.shape[2] != 2:
        raise ValueError("genotypes must have shape (variants, samples, 2)")
    a = g.astype(np.int16)
    if g.dtype == np.uint8:
        a = np.where(g == 255, -1, a)
    called = (a >= 0).all(axis=2)
    top = np.where(called, a.max(axis=2), -1).max(axis=1)
    if np.any(top > 3):
        raise ValueError("at most four alleles per site")
    multi = top >= 2
    codes = genotype_codes(g[~multi])
    with Estimator() as est:
        est.load(codes, allele_frequencies)
        if multi.any():
            am = a[multi]
            lo, hi = am.min(axis=2), am.max(axis=2)
            gi = np.where((am >= 0).all(axis=2), hi * (hi + 1) // 2 + lo, 255).astype(np.uint8)
            est.load_multiallelic(np.ascontiguousarray(gi.T), (top[multi] + 1).astype(np.uint8))
        if estimator == "ml":
            rows = est.relatedness(iterations=iterations)
        else:
            rows = est.relatedness_gt(iterations=iterations)
    return Coefficients(*build_arrays(rows, codes.shape[0]))


def read_vcf(path, field: str = "GT", allele_freqs: str = "estimate", threads: int = 0,
             multiallelic: bool = False, packed: bool = False):
    """Reads a plain, gzip or bgzip VCF with the library's multithreaded reader
    (the CLI's): biallelic SNP records become genotype codes.  Returns
    (codes u8 [samples, sites], allele_frequencies f64 [sites, 2] or None,
    sample names, counts dict).  allele_freqs "info" reads INFO/AF.  With
    multiallelic, a fifth item holds the tri- and tetra-allelic records:
    (genotype indices u8 [samples, sites] in the VCF order, 255 = missing,
    allele counts u8 [sites], allele frequencies f64 [sites, 4] or None), the
    arguments of Estimator.load_multiallelic.  With packed, codes is (2-bit codes,
    observed mask) as pack_2bit gives them, for Estimator.load_packed."""
    if allele_freqs not in ("estimate", "info"):
        raise ValueError("allele_freqs must be 'estimate' or 'info'")
    L = lib()
    h = ctypes.c_void_p()
    st = L.kg_vcf_read(os.fsencode(path), field.encode(), 1 if allele_freqs == "info" else 0, int(threads),
                       ctypes.byref(h))
    try:
        if st != KG_OK:
            msg = L.kg_vcf_error(h) if h.value else b"out of memory"
            raise KestrelError(st, msg.decode())
        ns, nv = ctypes.c_int64(), ctypes.c_int64()
        counts = (ctypes.c_uint64 * 7)()
        _check_vcf(L.kg_vcf_info(h, ctypes.byref(ns), ctypes.byref(nv), counts), L, h)
        af = np.empty((nv.value, 2)) if allele_freqs == "info" else None
        if packed:
            codes = (np.empty((ns.value, -(-nv.value // 16)), np.uint32),
                     np.empty((ns.value, -(-nv.value // 32)), np.uint32))
            _check_vcf(L.kg_vcf_codes_2bit(h, ptr(codes[0]), ptr(codes[1])), L, h)
            _check_vcf(L.kg_vcf_codes(h, None, ptr(af)), L, h)
        else:
            codes = np.empty((ns.value, nv.value), np.uint8)
            _check_vcf(L.kg_vcf_codes(h, ptr(codes), ptr(af)), L, h)
        names = [L.kg_vcf_sample(h, i).decode() for i in range(ns.value)]
        cd = {"sites": nv.value, "records": counts[0], "not_snp": counts[1], "multiallelic": counts[2],
              "soft_likelihoods": counts[3], "with_missing": counts[4], "tri_allelic": counts[5],
              "tetra_allelic": counts[6]}
        if not multiallelic:
            return codes, af, names, cd
        nm = counts[5] + counts[6]
        mg = np.empty((ns.value, nm), np.uint8)
        mal = np.empty(nm, np.uint8)
        maf = np.empty((nm, 4)) if allele_freqs == "info" else None
        _check_vcf(L.kg_vcf_multiallelic(h, ptr(mg), ptr(mal), ptr(maf)), L, h)
        return codes, af, names, cd, (mg, mal, maf)
    finally:
        if h.value:
            L.kg_vcf_free(h)


def read_vcf_likelihoods(path, field: str = "PL", threads: int = 0):
    """The linear-scale likelihoods of a GL/PL file's biallelic SNP records as
    the reference's reader makes them (10^(GL - max GL), 10^(-PL/10); NaN where
    missing), double [samples, sites, 3], the input of
    Estimator.load_likelihoods; None when every row is one-hot."""
    L = lib()
    h = ctypes.c_void_p()
    st = L.kg_vcf_read(os.fsencode(path), field.encode(), 0, int(threads), ctypes.byref(h))
    try:
        if st != KG_OK:
            msg = L.kg_vcf_error(h) if h.value else b"out of memory"
            raise KestrelError(st, msg.decode())
        ns, nv = ctypes.c_int64(), ctypes.c_int64()
        _check_vcf(L.kg_vcf_info(h, ctypes.byref(ns), ctypes.byref(nv), None), L, h)
        gl = np.empty((ns.value, nv.value, 3))
        st = L.kg_vcf_likelihoods(h, ptr(gl))
        if st == KG_ENOTFOUND:
            return None
        _check_vcf(st, L, h)
        return gl
    finally:
        if h.value:
            L.kg_vcf_free(h)


def _check_vcf(st, L, h):
    if st != KG_OK:
        raise KestrelError(st, L.kg_vcf_error(h).decode())


def relatedness_coefficients_gl(genotype_likelihoods, allele_frequencies=None, threads=None,
                                iterations=100, minimum_allele_frequency=None):
    """The GL/PL entry point (src/lib.rs:72-109) for biallelic likelihoods
    [variants, samples, 3] (linear scale, NaN = missing).  One-hot rows (to
    25.5 log10 units) go through the hard-call estimator (kg_relatedness); any
    other row sends the
    cohort through the soft-likelihood estimator (kg_relatedness_gl), which
    estimates the allele frequencies itself (the reference's GL path does not
    take given frequencies, src/wrapper.rs:118-126)."""
    del threads
    gl = np.asarray(genotype_likelihoods, dtype=np.float64)
    if gl.ndim != 3 or gl.shape[2] != 3:
        raise ValueError("genotype_likelihoods must have shape (variants, samples, 3)")
    miss = np.isnan(gl).any(axis=2)
    g = np.where(miss[..., None], 0.0, gl)
    best = np.argmax(g, axis=2)
    # one-hot to 25.5 log10 units (the reference's PL = 255 encoding leaves
    # 10^-25.5 residues, which move f, g and H by < 1e-18 relative)
    top = np.take_along_axis(g, best[..., None], axis=2)[..., 0]
    rest = np.sort(g, axis=2)[..., 1]
    soft = ~miss & (rest > top * 10 ** -25.5)
    if soft.any():
        if allele_frequencies is not None:
            raise ValueError("allele_frequencies cannot be given with soft likelihoods")
        with Estimator() as est:
            est.load_likelihoods(np.ascontiguousarray(gl.transpose(1, 0, 2)))
            rows = est.relatedness_gl(iterations=iterations, maf=minimum_allele_frequency)
        return build_arrays(rows, gl.shape[1])
    codes = best.astype(np.uint8)
    codes[miss] = MISSING
    codes = np.ascontiguousarray(codes.T)
    with Estimator() as est:
        est.load(codes, allele_frequencies)
        rows = est.relatedness(iterations=iterations, maf=minimum_allele_frequency)
    return build_arrays(rows, codes.shape[0])


def run_cli(argv=None) -> int:
    """`kestrel input.vcf kinship.tsv [flags]` (src/lib.rs:112-117, src/cli.rs:67-127)."""
    argv = list(sys.argv if argv is None else argv)
    L = lib()
    arr = (ctypes.c_char_p * len(argv))(*[a.encode() for a in argv])
    st = L.kg_run_cli(len(argv), arr)
    if st != 0:
        raise RuntimeError(f"kestrel exited with status {st}")
    return st
