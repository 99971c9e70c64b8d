"""The oracle's GL/PL estimator on soft genotype likelihoods (src/wrapper.rs:
89-330: the per-site allele-frequency SQP, zero-frequency alleles dropped,
pair rows sum over genotype pairs of GLx GLy m), checked against the hard-call
oracle on one-hot likelihoods and against numpy evaluations of its objectives.
CPU only."""
import numpy as np
import pytest

from kestrel_b200 import synth

from .test_oracle_cls import numpy_rows, row_index


def one_hot(codes):
    """codes [samples, sites] -> likelihoods [sites, samples, 3], NaN = missing."""
    gl = np.zeros(codes.T.shape + (3,))
    c = codes.T
    for g in range(3):
        gl[..., g] = c == g
    gl[c == synth.MISSING] = np.nan
    return gl


def soft_gl(codes, rng, err=0.05):
    """Likelihoods with mass off the called genotype, as sequencing gives."""
    gl = one_hot(codes)
    noise = rng.uniform(0, err, gl.shape)
    return np.where(np.isnan(gl), np.nan, np.where(gl == 1.0, 1.0, noise))


@pytest.fixture(scope="module")
def cohort():
    return synth.make_cohort(32, 2500, 31, missing=0.02,
                             planted={"parent_offspring": 3, "full_sib": 3}, name="gl")


def test_one_hot_likelihoods_give_the_hard_call_estimator(oracle, cohort):
    # maf away from 1 / (2 N): a fully called singleton's count frequency is
    # exactly 1 / (2 N), which the count form keeps and the SQP fit lands
    # within its tolerance of, on either side
    hard = oracle.relatedness(cohort.codes, maf=0.01)
    soft, af = oracle.gl_relatedness(one_hot(cohort.codes), maf=0.01)
    g = cohort.codes.astype(float)
    obs = cohort.codes < 3
    alt = np.where(obs, g, 0).sum(0) / (2 * obs.sum(0))
    seg = (alt > 0) & (alt < 1)
    assert np.abs(af[seg, 1] - alt[seg]).max() < 1e-6     # the SQP stops at KKT tolerance 1e-8
    lc = np.log10(hard["cond"])
    ident = np.isfinite(lc) & (lc < 15)
    # the frequencies differ at the SQP's tolerance, so the estimates at the
    # parity bar (Delta 1e-5 absolute, objective 1e-6 relative) and tighter
    assert np.abs(soft["jacquard"] - hard["jacquard"]).max(1)[ident].max() < 1e-6
    assert np.all(np.abs(soft["obj"] - hard["obj"]) <= 1e-7 * np.abs(hard["obj"]))
    assert np.mean(soft["iters"] == hard["iters"]) > 0.95


def af_objective(gl, x, eps=1e-8):
    a = len(x)
    p = np.full(gl.shape[0], eps)
    for j in range(a):
        for i in range(j + 1):
            w = x[i] * x[i] if i == j else 2 * x[i] * x[j]
            p += w * gl[:, j * (j + 1) // 2 + i]
    return -np.mean(np.log(p))


def test_allele_frequencies_are_optimal_on_the_simplex(oracle):
    rng = np.random.default_rng(9)
    for a, g in ((2, 3), (3, 6), (4, 10)):
        gl = rng.uniform(0.0, 1.0, (40, 200, g)) ** 3
        af = oracle.gl_allele_frequencies(gl, maf=0.0)
        for v in range(40):
            x = af[v, :a]
            assert abs(x.sum() - 1) < 1e-12 and np.all(x >= 0)
            f0 = af_objective(gl[v], x)
            # no feasible direction e_i - e_j (away from x_j > 0) decreases f
            for i in range(a):
                for j in range(a):
                    if i == j or x[j] <= 1e-9:
                        continue
                    h = min(1e-6, x[j])
                    d = np.zeros(a)
                    d[i] += h
                    d[j] -= h
                    assert af_objective(gl[v], x + d) >= f0 - 1e-9


def test_soft_pairs_against_numpy(oracle, cohort):
    rng = np.random.default_rng(10)
    gl = soft_gl(cohort.codes, rng)
    out, af = oracle.gl_relatedness(gl)
    keep = (af[:, 0] > 0) & (af[:, 1] > 0)
    p, q = af[keep, 0], af[keep, 1]
    M = numpy_rows(p, q)                         # [sites, gx, gy, 9]
    G = gl[keep]                                 # [sites, samples, 3]
    n = cohort.codes.shape[0]
    for x, y in [(0, 1), (3, 17), (5, 5), (30, 31)]:
        r = out[row_index(n, x, y)]
        rows = np.einsum("va,vb,vabk->vk", G[:, x], G[:, y], M)
        rows = rows[~np.isnan(rows).any(1)]
        d = r["jacquard"]
        e = rows @ d + 1e-8
        f = -np.mean(np.log(e))
        assert abs(f - r["obj"]) <= 1e-10 * abs(f)
        if x != y and r["iters"] < 100:
            grad = -(rows / e[:, None]).mean(0)
            lam = d @ grad
            viol = np.where(d > 0, np.abs(grad - lam), np.maximum(lam - grad, 0))
            assert viol.max() < 1e-7


def test_tri_site_with_an_absent_allele_is_biallelic(oracle, cohort):
    rng = np.random.default_rng(11)
    gl = soft_gl(cohort.codes, rng)
    cut = 2000
    base, af = oracle.gl_relatedness(gl)
    tri = np.zeros((gl.shape[0] - cut, gl.shape[1], 6))
    tri[..., :3] = gl[cut:]                      # genotypes with allele 2 are impossible
    tri[np.isnan(gl[cut:]).any(2)] = np.nan
    split, af2 = oracle.gl_relatedness(gl[:cut], gl3=tri)
    assert np.all(af2[cut:, 2] == 0.0)
    assert np.abs(af2[cut:, :2] - af[cut:, :2]).max() < 1e-7
    lc = np.log10(base["cond"])
    ident = np.isfinite(lc) & (lc < 15)
    assert np.abs(split["jacquard"] - base["jacquard"]).max(1)[ident].max() < 1e-6
    assert np.all(np.abs(split["obj"] - base["obj"]) <= 1e-9 * np.abs(base["obj"]))


def test_singleton_at_the_default_maf_sits_on_the_cut(oracle, cohort):
    # the default maf is 1 / (2 N); the SQP puts a fully called singleton's
    # frequency within 1e-6 of it, where the cut drops it or not
    codes = cohort.codes.copy()
    codes[:, 0] = 0
    codes[0, 0] = 1                               # one ALT allele in 64
    _, af = oracle.gl_relatedness(one_hot(codes[:, :50]))
    n = codes.shape[0]
    assert af[0, 1] == 0.0 or abs(af[0, 1] - 1 / (2 * n)) < 1e-6


def test_device_allele_fit_matches_the_oracle(oracle, tmp_path):
    """The GPU's per-site frequency fit for 2-4 alleles (kg_alleleN.cuh, the
    class-count form of the reference's allele SQP on one-hot likelihoods),
    built for the host, against the oracle's fit of the same calls given as
    per-sample one-hot rows: equal to 1e-7 (the two sum in different orders,
    so the SQP can stop an iterate apart within its KKT tolerance of 1e-8),
    with the same frequencies cut to zero by maf."""
    import os
    import shutil
    import subprocess
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = str(tmp_path / "allele_fit_host")
    subprocess.run([nvcc, "-O2", "-std=c++17", "-I", os.path.join(root, "kestrel_b200", "csrc"),
                    os.path.join(root, "tests", "host", "allele_fit_host.cu"), "-o", exe], check=True)
    rng = np.random.default_rng(5)
    lines, cases = [], []
    for a in (2, 3, 4):
        ng = a * (a + 1) // 2
        for k in range(60):
            n = int(rng.integers(5, 200))
            f = rng.dirichlet(np.full(a, 0.6))
            al = rng.choice(a, size=(n, 2), p=f)
            i, j = al.min(1), al.max(1)
            g = j * (j + 1) // 2 + i
            if k % 7 == 0:
                g[rng.random(n) < 0.2] = ng                       # missing
            cnt = np.bincount(g[g < ng], minlength=ng)
            maf = 1.0 / (2 * n) if k % 2 else 0.02
            lines.append(f"{a} " + " ".join(str(c) for c in cnt) + f" 100 {maf!r}")
            gl = np.zeros((1, n, ng))
            for c in range(ng):
                gl[0, :, c] = g == c
            gl[0, g == ng] = np.nan
            cases.append((a, gl, maf))
    out = subprocess.run([exe], input=f"{len(lines)}\n" + "\n".join(lines) + "\n", capture_output=True,
                         text=True, check=True).stdout.split("\n")
    worst = 0.0
    for (a, gl, maf), line in zip(cases, out):
        got = np.array([float(v) for v in line.split()])[:a]
        want = oracle.gl_allele_frequencies(gl, maf=maf)[0, :a]
        assert np.array_equal(got > 0, want > 0), (a, got, want)
        worst = max(worst, float(np.abs(got - want).max()))
        assert np.abs(got - want).max() <= 1e-7, (a, got, want)
    print("largest frequency difference", worst)
