"""The multithreaded VCF reader (kg_vcf_read; the CLI's reader) against a plain
Python parser written from the same record rules: plain, gzip and bgzip input,
GT/PL/GL fields, skipped records, INFO/AF, thread-count invariance, and the
first error in file order.  CPU only."""
import gzip
import os
import struct
import tempfile
import zlib

import numpy as np
import pytest

import kestrel_b200 as kb
from kestrel_b200 import synth

BASES = set("ACGTacgt")


def py_parse(text, field="GT", af_info=False):
    """Reference parse: returns (codes [S, V], af or None, samples, counts,
    (multi-allelic genotype indices [S, Vm], allele counts, af [Vm, 4] or None))."""
    key = field
    samples, rows, afs = [], [], []
    mrows, malleles, mafs = [], [], []
    total = not_snp = multi = soft = with_missing = tri = tetra = 0
    for line in text.split("\n"):
        line = line.rstrip("\r")
        if line.startswith("#CHROM"):
            samples = line.split("\t")[9:]
            continue
        if not line or line.startswith("#"):
            continue
        total += 1
        cols = line.split("\t")
        if len(cols) < 9 + len(samples) or not samples:
            raise ValueError(f"malformed record {total}")
        alts = cols[4].split(",")
        snp = len(cols[3]) == 1 and cols[3] in BASES and all(len(a) == 1 and a in BASES for a in alts)
        nb = len(alts) + 1
        if not snp or nb > 4:
            not_snp += 1
            continue
        if nb > 2:
            multi += 1
        fmt = cols[8].split(":")
        fi = max([i for i, f in enumerate(fmt) if f == key], default=-1)
        if fi < 0:
            raise ValueError(f"No {key} data found")

        def value(s):
            sub = cols[9 + s].split(":")
            return sub[fi] if fi < len(sub) else "."
        if nb > 2:
            # every record kept, a missing call as 255; GT: a malformed call
            # after a missing one drops the record (the reference's reader
            # stops at the missing call); GL/PL: the most likely genotype
            row, missing, dropped = [], False, False
            ng = nb * (nb + 1) // 2
            for s in range(len(samples)):
                v = value(s)
                if field == "GT":
                    parts = v.replace("|", "/").split("/")
                    if "." in parts and len(parts) <= 2:
                        missing = True
                        row.append(255)
                        continue
                    if len(parts) != 2 or not all(p.isdigit() and int(p) < nb for p in parts):
                        if missing:
                            dropped = True
                            break
                        raise ValueError(f"Value {v} is not a valid GT")
                    i, j = sorted(int(p) for p in parts)
                    row.append(j * (j + 1) // 2 + i)
                else:
                    parts = v.split(",")
                    if v != "." and len(parts) != ng:
                        raise ValueError(f"Value {v} is not a valid {key}")
                    if v == "." or "." in parts:
                        missing = True
                        row.append(255)
                        continue
                    val = [float(p) for p in parts]
                    ll = [-x / 10.0 for x in val] if field == "PL" else val
                    row.append(int(np.argmax(ll)))
            if missing:
                with_missing += 1
            if dropped:
                continue
            if af_info:
                vals = None
                for kv in cols[7].split(";"):
                    if kv.startswith("AF="):
                        vals = [float(x) for x in kv[3:].split(",")]
                if vals is None:
                    raise ValueError("No AF info found")
                if len(vals) != nb - 1:
                    raise ValueError("allele frequencies")
                alt_sum = 0.0
                for x in vals:          # in order, as the reference adds them
                    alt_sum += x
                f = [1.0 - min(max(alt_sum, 0.0), 1.0)] + vals
                mafs.append(f + [0.0] * (4 - len(f)))
            mrows.append(row)
            malleles.append(nb)
            tri += nb == 3
            tetra += nb == 4
            continue
        row = []
        for s in range(len(samples)):
            v = value(s)
            if field == "GT":
                parts = v.replace("|", "/").split("/")
                if "." in parts:
                    if len(parts) > 2:
                        raise ValueError(f"Value {v} is not a valid GT")
                    row.append(3)
                    continue
                if len(parts) != 2 or not all(p in ("0", "1") for p in parts):
                    raise ValueError(f"Value {v} is not a valid GT")
                row.append(int(parts[0]) + int(parts[1]))
            else:
                if v == ".":
                    row.append(3)
                    continue
                parts = v.split(",")
                if len(parts) != 3:
                    raise ValueError(f"Value {v} is not a valid {key}")
                if "." in parts:
                    row.append(3)
                    continue
                val = [float(p) for p in parts]
                ll = [-x / 10.0 for x in val] if field == "PL" else val
                best = int(np.argmax(ll))
                if any(i != best and ll[best] - ll[i] < 25.5 - 1e-9 for i in range(3)):
                    soft += 1
                row.append(best)
        if af_info:
            a = float("nan")
            for kv in cols[7].split(";"):
                if kv.startswith("AF="):
                    a = float(kv[3:].split(",")[0])
            if np.isnan(a):
                raise ValueError("No AF info found")
            afs.append([1.0 - min(max(a, 0.0), 1.0), a])
        with_missing += 3 in row
        rows.append(row)
    ns = len(samples)
    codes = np.array(rows, np.uint8).T.reshape(ns, len(rows)) if rows else np.zeros((ns, 0), np.uint8)
    mg = np.array(mrows, np.uint8).T.reshape(ns, len(mrows)) if mrows else np.zeros((ns, 0), np.uint8)
    counts = {"sites": len(rows), "records": total, "not_snp": not_snp, "multiallelic": multi, "soft_likelihoods": soft,
              "with_missing": with_missing, "tri_allelic": tri, "tetra_allelic": tetra}
    return codes, (np.array(afs) if af_info else None), samples, counts, \
        (mg, np.array(malleles, np.uint8), (np.array(mafs).reshape(-1, 4) if af_info else None))


def write_bgzip(path, data: bytes, block=65280):
    """BGZF: gzip members of at most 64 KB with the 'BC' extra subfield, then the
    empty end-of-file member."""
    with open(path, "wb") as fh:
        for i in range(0, len(data) + 1, block):
            chunk = data[i:i + block]
            if not chunk and i:
                break
            co = zlib.compressobj(6, zlib.DEFLATED, -15)
            comp = co.compress(chunk) + co.flush()
            bsize = 18 + len(comp) + 8 - 1
            fh.write(b"\x1f\x8b\x08\x04\x00\x00\x00\x00\x00\xff\x06\x00BC\x02\x00" + struct.pack("<H", bsize))
            fh.write(comp)
            fh.write(struct.pack("<II", zlib.crc32(chunk) & 0xffffffff, len(chunk)))
        fh.write(bytes.fromhex("1f8b08040000000000ff0600424302001b0003000000000000000000"))


def edge_records(n):
    def calls(txt):
        return "\t".join([txt] * n)

    def mixed(*txt):
        return "\t".join(txt[i % len(txt)] for i in range(n))
    return [f"2\t1\t.\tA\tC,G\t.\tPASS\tAF=0.2,0.1\tGT\t{mixed('0/1', '2/2', '1|2', '0/0')}",  # tri-allelic
            f"2\t2\t.\tAT\tC\t.\tPASS\tAF=0.2\tGT\t{calls('0/1')}",       # not a SNP
            f"2\t3\t.\tG\t<DEL>\t.\tPASS\tAF=0.2\tGT\t{calls('1/1')}",    # symbolic ALT
            f"2\t4\t.\tT\tG\t.\tPASS\tAF=0.4;DP=9\tGT:DP\t{calls('0|1:7')}",
            f"2\t5\t.\tc\tg\t.\tPASS\tDP=3;AF=0.7\tDP:GT\t{calls('5:1/1')}",
            f"2\t6\t.\tA\tT\t.\tPASS\tAF=0.5\tGT\t{calls('./.')}",
            f"2\t7\t.\tA\tC,G,T\t.\tPASS\tAF=0.1,0.2,0.3\tGT\t{mixed('3/1', '0/3', '2/2', '1/1')}",  # tetra
            f"2\t8\t.\tA\tC,G\t.\tPASS\tAF=0.2,0.1\tGT\t{mixed('0/1', './.', '2/9')}",  # missing: skipped
            f"2\t9\t.\tA\tC,G,T,A\t.\tPASS\tAF=0.1,0.1,0.1,0.1\tGT\t{calls('0/1')}"]   # five bases


@pytest.fixture(scope="module")
def cohort():
    return synth.make_cohort(37, 3000, 61, missing=0.03, name="vcf")


def make_text(codes, field, extra=True, crlf=False):
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "x.vcf")
        synth.write_vcf(p, codes, field=field)
        text = open(p).read()
    text = text.replace("\tPASS\t.\t", "\tPASS\tAF=0.25\t")
    if extra and field == "GT":
        text += "\n".join(edge_records(codes.shape[0])) + "\n"
    if crlf:
        text = text.replace("\n", "\r\n")
    return text


@pytest.mark.parametrize("compression", ["plain", "gzip", "bgzip"])
@pytest.mark.parametrize("field", ["GT", "PL"])
def test_reader_matches_python(cohort, field, compression):
    text = make_text(cohort.codes, field)
    ref = py_parse(text, field, af_info=True)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "x.vcf" + ("" if compression == "plain" else ".gz"))
        data = text.encode()
        if compression == "plain":
            open(p, "wb").write(data)
        elif compression == "gzip":
            with gzip.open(p, "wb") as fh:
                fh.write(data)
        else:
            write_bgzip(p, data)
        for threads in (1, 3, 8):
            codes, af, names, counts, multi = kb.read_vcf(p, field, allele_freqs="info", threads=threads,
                                                          multiallelic=True)
            assert np.array_equal(codes, ref[0])
            assert np.array_equal(af, ref[1])
            assert names == ref[2]
            assert counts == ref[3]
            for a, b in zip(multi, ref[4]):
                assert np.array_equal(a, b)
    if field == "GT":
        assert counts["multiallelic"] == 3 and counts["not_snp"] == 3
        assert counts["tri_allelic"] == 1 and counts["tetra_allelic"] == 1
        assert multi[0][:4, 1].tolist() == [7, 6, 5, 2]   # 3/1, 0/3, 2/2, 1/1


def test_crlf_and_gl_field(cohort):
    gl = np.array(["0,-25.5,-30", "-26,0,-40", "-50,-30,0", "."])
    lines = ["##fileformat=VCFv4.2", "#CHROM\tPOS\tID\tREF\tALT\tQUAL\tFILTER\tINFO\tFORMAT\tA\tB\tC"]
    rng = np.random.default_rng(2)
    for s in range(200):
        c = rng.integers(0, 4, 3)
        lines.append(f"1\t{s + 1}\t.\tA\tG\t.\tPASS\t.\tGL\t" + "\t".join(gl[c]))
    text = "\r\n".join(lines) + "\r\n"
    ref = py_parse(text, "GL")
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "gl.vcf")
        open(p, "w", newline="").write(text)
        codes, _, names, counts = kb.read_vcf(p, "GL", threads=4)
    assert names == ["A", "B", "C"]
    assert np.array_equal(codes, ref[0]) and counts == ref[3]


def test_multichunk_first_error_in_file_order():
    # a body above 1 MB is cut into chunks; the first bad record (file order)
    # is reported with its global record number
    co = synth.make_cohort(64, 12000, 62, missing=0.01, name="big")
    text = make_text(co.codes, "GT", extra=False)
    lines = text.split("\n")
    body = [i for i, ln in enumerate(lines) if ln and not ln.startswith("#")]
    bad1, bad2 = body[7000], body[9000]
    lines[bad2] = lines[bad2].replace("0/0", "0/7", 1).replace("0/1", "0/7", 1).replace("1/1", "0/7", 1)
    lines[bad1] = "\t".join(lines[bad1].split("\t")[:20])   # too few columns
    bad_text = "\n".join(lines)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "bad.vcf")
        open(p, "w").write(bad_text)
        assert len(bad_text) > (1 << 20)
        for threads in (1, 8):
            with pytest.raises(kb.KestrelError, match="malformed record 7001"):
                kb.read_vcf(p, "GT", threads=threads)
        good = os.path.join(td, "good.vcf")
        open(good, "w").write(text)
        codes, _, _, counts = kb.read_vcf(good, "GT", threads=8)
        assert np.array_equal(codes, co.codes) and counts["records"] == 12000


def test_reader_errors(cohort):
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "x.vcf")
        open(p, "w").write("##fileformat=VCFv4.2\n#CHROM\tPOS\tID\tREF\tALT\tQUAL\tFILTER\tINFO\tFORMAT\tA\n"
                           "1\t1\t.\tA\tC\t.\tPASS\t.\tDP\t3\n")
        with pytest.raises(kb.KestrelError, match="No GT data found"):
            kb.read_vcf(p, "GT")
        with pytest.raises(kb.KestrelError, match="No AF info found"):
            open(p, "w").write("#CHROM\tPOS\tID\tREF\tALT\tQUAL\tFILTER\tINFO\tFORMAT\tA\n"
                               "1\t1\t.\tA\tC\t.\tPASS\t.\tGT\t0/1\n")
            kb.read_vcf(p, "GT", allele_freqs="info")
        with pytest.raises(kb.KestrelError, match="cannot open"):
            kb.read_vcf(os.path.join(td, "missing.vcf"))
        with pytest.raises(kb.KestrelError, match="field must be"):
            kb.read_vcf(p, "XX")


def test_fifo_input_is_read_without_mapping(cohort):
    # a pipe cannot be mapped: the reader falls back to reading it
    import threading
    text = make_text(cohort.codes, "GT")
    ref = py_parse(text, "GT")
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "pipe.vcf")
        os.mkfifo(p)

        def feed():
            with open(p, "w") as fh:
                fh.write(text)
        th = threading.Thread(target=feed)
        th.start()
        codes, _, names, counts = kb.read_vcf(p, "GT", threads=4)
        th.join()
    assert np.array_equal(codes, ref[0]) and names == ref[2] and counts == ref[3]


def test_packed_codes_decode_to_the_byte_codes():
    co = synth.make_cohort(21, 3001, 63, missing=0.05, name="packed")   # ragged last words
    text = make_text(co.codes, "GT", extra=False)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "x.vcf")
        open(p, "w").write(text)
        (c2, ob), _, _, _ = kb.read_vcf(p, "GT", packed=True, threads=3)
        codes, _, _, _ = kb.read_vcf(p, "GT")
    assert np.array_equal(codes, co.codes)
    n2, nm = kb.pack_2bit(codes)
    assert np.array_equal(c2, n2) and np.array_equal(ob, nm)
    s = np.arange(codes.shape[1])
    dec = (c2[:, s // 16] >> (2 * (s % 16)).astype(np.uint32)) & 3
    obs = (ob[:, s // 32] >> (s % 32).astype(np.uint32)) & 1
    assert np.array_equal(np.where(obs == 1, dec, 3), codes)


def soft_pl_text(codes, rng):
    """A PL VCF whose rows are not one-hot: 0 at the call, 5-40 elsewhere."""
    n, m = codes.shape
    lines = ["##fileformat=VCFv4.2", "#CHROM\tPOS\tID\tREF\tALT\tQUAL\tFILTER\tINFO\tFORMAT\t" +
             "\t".join(f"S{i}" for i in range(n))]
    for v in range(m):
        calls = []
        for s in range(n):
            c = codes[s, v]
            if c == 3:
                calls.append(".,.,.")
                continue
            pl = rng.integers(5, 41, 3)
            pl[c] = 0
            calls.append(",".join(str(x) for x in pl))
        lines.append(f"1\t{v + 1}\t.\tA\tC\t.\tPASS\t.\tPL\t" + "\t".join(calls))
    return "\n".join(lines) + "\n"


def py_likelihoods(text, field):
    samples, rows = None, []
    for line in text.split("\n"):
        if line.startswith("#CHROM"):
            samples = line.split("\t")[9:]
        if not line or line.startswith("#"):
            continue
        cols = line.split("\t")
        row = []
        for v in cols[9:9 + len(samples)]:
            parts = v.split(",")
            if "." in parts:
                row.append([np.nan] * 3)
            elif field == "PL":
                row.append([10.0 ** (-float(x) / 10.0) for x in parts])
            else:
                g = [float(np.float32(float(x))) for x in parts]
                mx = max(g)
                row.append([10.0 ** (x - mx) for x in g])
        rows.append(row)
    return np.array(rows).transpose(1, 0, 2)


def test_soft_likelihoods_are_read_as_the_reference_makes_them():
    co = synth.make_cohort(19, 900, 64, missing=0.03, name="soft-pl")
    text = soft_pl_text(co.codes, np.random.default_rng(1))
    gl_text = text.replace("\tPL\t", "\tGL\t")   # the same numbers read as GL (log10 scale)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "pl.vcf")
        open(p, "w").write(text)
        g = os.path.join(td, "gl.vcf")
        open(g, "w").write(gl_text)
        got = kb.read_vcf_likelihoods(p, "PL", threads=3)
        got_gl = kb.read_vcf_likelihoods(g, "GL", threads=3)
        hard = os.path.join(td, "hard.vcf")
        synth.write_vcf(hard, co.codes, field="PL")
        assert kb.read_vcf_likelihoods(hard, "PL") is None     # one-hot: no likelihoods kept
    want = py_likelihoods(text, "PL")
    assert np.array_equal(np.isnan(got), np.isnan(want))
    assert np.allclose(got, want, rtol=1e-15, atol=0, equal_nan=True)
    want_gl = py_likelihoods(gl_text, "GL")
    assert np.allclose(got_gl, want_gl, rtol=1e-15, atol=0, equal_nan=True)


def test_likelihood_fields_keep_multiallelic_records():
    """GL/PL tri- and tetra-allelic records are kept (the ML estimator's input):
    each call becomes its most likely genotype in the VCF order, a missing value
    or entry 255; rows that are not one-hot count apart from the biallelic ones."""
    rng = np.random.default_rng(8)
    n = 6
    lines = ["##fileformat=VCFv4.2", "#CHROM\tPOS\tID\tREF\tALT\tQUAL\tFILTER\tINFO\tFORMAT\t" +
             "\t".join(f"S{i}" for i in range(n))]
    for v in range(40):
        nb = int(rng.integers(2, 5))
        ng = nb * (nb + 1) // 2
        alt = ",".join("CGT"[:nb - 1])
        calls = []
        for s in range(n):
            r = rng.random()
            if r < 0.1:
                calls.append(".")
            elif r < 0.15:
                calls.append(",".join("." if k == 1 else "0" for k in range(ng)))
            else:
                pl = np.full(ng, 255)
                pl[int(rng.integers(0, ng))] = 0
                if r > 0.9:
                    pl[int(rng.integers(0, ng))] = 7        # not one-hot
                calls.append(",".join(str(int(x)) for x in pl))
        lines.append(f"3\t{v + 1}\t.\tA\t{alt}\t.\tPASS\t.\tPL\t" + "\t".join(calls))
    text = "\n".join(lines) + "\n"
    ref = py_parse(text, "PL")
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "pl.vcf")
        open(p, "w").write(text)
        for threads in (1, 4):
            codes, _, _, counts, multi = kb.read_vcf(p, "PL", threads=threads, multiallelic=True)
            assert np.array_equal(codes, ref[0])
            for a, b in zip(multi[:2], ref[4][:2]):
                assert np.array_equal(a, b)
            assert counts["tri_allelic"] == ref[3]["tri_allelic"] > 0
            assert counts["tetra_allelic"] == ref[3]["tetra_allelic"] > 0
            assert counts["with_missing"] == ref[3]["with_missing"]
    assert np.any(ref[4][0] == 255)
