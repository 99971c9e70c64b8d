"""Seeded synthetic cohorts for the relatedness estimator.

There is no public dataset for this path (the reference validates on msprime
pedigree simulations and Ag3 mosquito data, neither present here), so the
workloads are generated with the shapes and distributions the benchmark
configurations describe:

* per site, the REF allele frequency p ~ Beta(0.5, 0.5) clipped to [0.05, 0.95];
* genotypes (ALT allele counts 0/1/2) under Hardy-Weinberg;
* calls set missing independently (code 3);
* related pairs planted by drawing, per site, a Jacquard state from the pair's
  Delta and the four alleles from that state's identity-by-descent partition.

Genotype codes follow the reference's unphased triangular index
(src/coefficients.rs:19-38): 0 = 0/0, 1 = 0/1, 2 = 1/1, and 3 marks a missing
call (the reference's NaN likelihood, src/vcf.rs:397).  Arrays are sample-major
(n_samples, n_sites) uint8.
"""
from __future__ import annotations

import dataclasses

import numpy as np

MISSING = 3

# Identity-by-descent partitions of the four alleles (x1, x2, y1, y2) for the
# nine condensed Jacquard states, as class labels per allele.
_STATE_CLASSES = np.array(
    [
        [0, 0, 0, 0],  # S1: all four IBD
        [0, 0, 1, 1],  # S2: x autozygous, y autozygous, not IBD across
        [0, 0, 0, 1],  # S3: x autozygous, one allele of y IBD to it
        [0, 0, 1, 2],  # S4: x autozygous, y not, nothing across
        [0, 1, 0, 0],  # S5: y autozygous, one allele of x IBD to it
        [0, 1, 2, 2],  # S6: y autozygous, x not, nothing across
        [0, 1, 0, 1],  # S7: both alleles IBD across
        [0, 1, 0, 2],  # S8: one allele IBD across
        [0, 1, 2, 3],  # S9: nothing IBD
    ],
    dtype=np.int8,
)

PLANTED_DELTAS = {
    "parent_offspring": np.array([0, 0, 0, 0, 0, 0, 0, 1.0, 0]),
    "full_sib": np.array([0, 0, 0, 0, 0, 0, 0.25, 0.5, 0.25]),
    "half_sib": np.array([0, 0, 0, 0, 0, 0, 0, 0.5, 0.5]),
    "first_cousin": np.array([0, 0, 0, 0, 0, 0, 0, 0.25, 0.75]),
    "identical_inbred": np.array([1.0, 0, 0, 0, 0, 0, 0, 0, 0]),
}


@dataclasses.dataclass
class Cohort:
    codes: np.ndarray            # (n_samples, n_sites) uint8, 3 = missing
    p_true: np.ndarray           # (n_sites,) generating REF frequency
    planted: list                # [(x, y, name, delta[9])]
    seed: int
    name: str = ""

    @property
    def n_samples(self) -> int:
        return self.codes.shape[0]

    @property
    def n_sites(self) -> int:
        return self.codes.shape[1]


def site_frequencies(rng: np.random.Generator, n_sites: int) -> np.ndarray:
    p = rng.beta(0.5, 0.5, size=n_sites)
    return np.clip(p, 0.05, 0.95)


def _alt_alleles(rng, q, shape):
    """Bernoulli(q) ALT indicators, q broadcast over the trailing (site) axis."""
    u = rng.random(shape, dtype=np.float32)
    return (u < q.astype(np.float32)).astype(np.uint8)


def hwe_genotypes(rng: np.random.Generator, p: np.ndarray, n: int,
                  inbreeding: np.ndarray | None = None) -> np.ndarray:
    """(n, n_sites) ALT counts under HWE; rows with inbreeding F are autozygous
    at each site with probability F."""
    q = 1.0 - p
    a1 = _alt_alleles(rng, q, (n, p.size))
    a2 = _alt_alleles(rng, q, (n, p.size))
    if inbreeding is not None:
        auto = rng.random((n, p.size), dtype=np.float32) < \
            np.asarray(inbreeding, dtype=np.float32)[:, None]
        a2 = np.where(auto, a1, a2)
    return a1 + a2


def pair_genotypes(rng: np.random.Generator, p: np.ndarray, delta: np.ndarray):
    """Genotypes of one related pair: per site a Jacquard state ~ Categorical(delta)
    and the four alleles drawn from that state's IBD partition."""
    m = p.size
    q = (1.0 - p).astype(np.float32)
    delta = np.asarray(delta, dtype=np.float64)
    delta = delta / delta.sum()
    states = rng.choice(9, size=m, p=delta)
    classes = _STATE_CLASSES[states]                       # (m, 4)
    draws = (rng.random((m, 4), dtype=np.float32) < q[:, None]).astype(np.uint8)
    alleles = np.take_along_axis(draws, classes.astype(np.int64), axis=1)
    gx = alleles[:, 0] + alleles[:, 1]
    gy = alleles[:, 2] + alleles[:, 3]
    return gx.astype(np.uint8), gy.astype(np.uint8)


def apply_missing(rng, codes, rate):
    """Set calls missing independently; rate is a scalar or a per-sample vector."""
    rate = np.asarray(rate, dtype=np.float32)
    if rate.ndim == 1:
        rate = rate[:, None]
    miss = rng.random(codes.shape, dtype=np.float32) < rate
    codes[miss] = MISSING
    return codes


def make_cohort(n_samples: int, n_sites: int, seed: int, missing=0.02,
                planted: dict | None = None, inbred: int = 0,
                inbred_f=(0.0625, 0.25), low_info_sites: int = 0,
                name: str = "") -> Cohort:
    """A cohort with optional planted pairs (name -> count), inbred individuals
    and a block of low-information sites (p in [0.45, 0.55])."""
    rng = np.random.default_rng(seed)
    p = site_frequencies(rng, n_sites)
    if low_info_sites:
        idx = rng.choice(n_sites, size=low_info_sites, replace=False)
        p[idx] = rng.uniform(0.45, 0.55, size=low_info_sites)
    n_pairs = sum((planted or {}).values())
    assert 2 * n_pairs + inbred <= n_samples, "not enough samples for the plan"
    order = rng.permutation(n_samples)
    f = np.zeros(n_samples)
    inbred_ids = order[2 * n_pairs: 2 * n_pairs + inbred]
    f[inbred_ids] = rng.uniform(inbred_f[0], inbred_f[1], size=inbred)
    codes = hwe_genotypes(rng, p, n_samples, inbreeding=f if inbred else None)
    plan = []
    k = 0
    for rel, count in (planted or {}).items():
        for _ in range(count):
            a, b = int(order[2 * k]), int(order[2 * k + 1])
            gx, gy = pair_genotypes(rng, p, PLANTED_DELTAS[rel])
            codes[a] = gx
            codes[b] = gy
            plan.append((min(a, b), max(a, b), rel,
                         PLANTED_DELTAS[rel] if a < b else swap_xy(PLANTED_DELTAS[rel])))
            k += 1
    apply_missing(rng, codes, missing)
    return Cohort(codes=codes, p_true=p, planted=plan, seed=seed, name=name)


def make_multiallelic(n_samples: int, n_sites: int, seed: int, missing: float = 0.0):
    """Tri- and tetra-allelic sites under Hardy-Weinberg proportions:
    (genotype indices u8 [samples, sites] in the VCF order j (j + 1) / 2 + i,
    255 = missing; allele counts u8 [sites], 3 or 4)."""
    rng = np.random.default_rng(seed)
    al = rng.integers(3, 5, n_sites).astype(np.uint8)
    g = np.zeros((n_samples, n_sites), np.uint8)
    for v in range(n_sites):
        f = rng.dirichlet(np.full(int(al[v]), 0.8))
        a = rng.choice(int(al[v]), size=(n_samples, 2), p=f)
        i, j = a.min(1), a.max(1)
        g[:, v] = j * (j + 1) // 2 + i
    if missing > 0:
        g[rng.random(g.shape) < missing] = 255
    return g, al


def swap_xy(delta):
    """Delta of (y, x) from Delta of (x, y): D3<->D5 and D4<->D6 (src/lib.rs:138-149)."""
    d = np.array(delta, dtype=np.float64)
    return d[[0, 1, 4, 5, 2, 3, 6, 7, 8]]


# ------------------------------------------------------------- configurations

def config0(seed: int = 0) -> Cohort:
    """N=64 x M=10,000, 2% missing: the CPU-runnable plain case."""
    return make_cohort(64, 10_000, seed, name="cfg0")


def config1(seed: int = 1, n_samples: int = 1024, n_sites: int = 100_000) -> Cohort:
    """N=1024 x M=100,000 with 64 each of PO, FS, HS and FC pairs planted (fewer,
    n_samples // 16 each, for smaller test cohorts)."""
    k = min(64, n_samples // 16)
    return make_cohort(n_samples, n_sites, seed,
                       planted={"parent_offspring": k, "full_sib": k,
                                "half_sib": k, "first_cousin": k},
                       name="cfg1")


CONFIG2_SAMPLES = (96, 160, 256, 384, 512, 768, 1024, 2048)
CONFIG2_SITES = (20_000, 35_000, 50_000, 65_000, 80_000, 90_000, 95_000, 100_000)


def config2(seed: int = 2, scale: float = 1.0) -> list:
    """Eight uneven cohorts with per-sample missingness ~ U(0, 0.2).  scale < 1
    shrinks both axes for quick tests."""
    out = []
    for i, (n, m) in enumerate(zip(CONFIG2_SAMPLES, CONFIG2_SITES)):
        n = max(4, int(round(n * scale)))
        m = max(64, int(round(m * scale)))
        rng = np.random.default_rng(seed * 1000 + i)
        rate = rng.uniform(0.0, 0.2, size=n)
        out.append(make_cohort(n, m, seed * 1000 + i + 1, missing=rate, name=f"cfg2.{i}"))
    return out


def config3(seed: int = 3, n_samples: int = 512, n_sites: int = 50_000) -> Cohort:
    """N=512 x M=50,000: 128 inbred individuals, 32 identical-inbred pairs and a
    5,000-site low-information block."""
    return make_cohort(n_samples, n_sites, seed, planted={"identical_inbred": 32},
                       inbred=128, low_info_sites=n_sites // 10, name="cfg3")


def config4_panel(seed: int = 4, n_samples: int = 4096, n_sites: int = 100_000) -> Cohort:
    """Serving panel: 4,096 x 100,000 built as config 0."""
    return make_cohort(n_samples, n_sites, seed, name="cfg4")


def config4_requests(panel: Cohort, n_requests: int, seed: int = 44, rate_hz: float = 200.0,
                     max_query: int = 64):
    """Poisson arrivals of query batches: 1..max_query new samples drawn like the
    panel, each request keeping a random U(0.6, 1.0) fraction of sites."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate_hz, size=n_requests))
    reqs = []
    for i in range(n_requests):
        nq = int(rng.integers(1, max_query + 1))
        codes = hwe_genotypes(rng, panel.p_true, nq)
        apply_missing(rng, codes, 0.02)
        keep = rng.random(panel.n_sites) < rng.uniform(0.6, 1.0)
        reqs.append({"arrival_s": float(t[i]), "codes": codes, "site_mask": keep})
    return reqs


# ------------------------------------------------------------------ VCF output

def write_vcf(path, codes: np.ndarray, field: str = "GT", sample_names=None,
              chrom: str = "1", alleles=("A", "C")) -> None:
    """Writes a VCF 4.2 file of biallelic SNPs with either hard calls (GT) or the
    equivalent one-hot phred likelihoods (PL: 0 at the call, 255 elsewhere, '.'
    when missing).  Used to drive the CLI on synthetic cohorts."""
    n, m = codes.shape
    names = sample_names or [f"S{i}" for i in range(n)]
    gt_txt = np.array(["0/0", "0/1", "1/1", "./."])
    pl_txt = np.array(["0,255,255", "255,0,255", "255,255,0", ".,.,."])
    with open(path, "w") as fh:
        fh.write("##fileformat=VCFv4.2\n")
        fh.write(f"##contig=<ID={chrom}>\n")
        if field == "GT":
            fh.write('##FORMAT=<ID=GT,Number=1,Type=String,Description="Genotype">\n')
        else:
            fh.write('##FORMAT=<ID=PL,Number=G,Type=Integer,Description="Phred-scaled likelihoods">\n')
        fh.write("#CHROM\tPOS\tID\tREF\tALT\tQUAL\tFILTER\tINFO\tFORMAT\t" + "\t".join(names) + "\n")
        table = gt_txt if field == "GT" else pl_txt
        for s in range(m):
            calls = "\t".join(table[codes[:, s]])
            fh.write(f"{chrom}\t{s + 1}\t.\t{alleles[0]}\t{alleles[1]}\t.\tPASS\t.\t{field}\t{calls}\n")
