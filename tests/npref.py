"""Independent numpy evaluation of the ML objective, gradient and Hessian
(test helper).  Builds the nine one-hot likelihood rows from the conditional
genotype-pair table of the reference (src/iis.rs:279-462, two-allele case) in
closed form, without sharing code with the C oracle or the CUDA kernels."""
import numpy as np


def likelihood_rows(gx, gy, p, q):
    """(n, 9) rows P(gx, gy | S_k) for hard calls gx, gy in {0,1,2}."""
    n = gx.size
    L = np.zeros((n, 9))
    # probability that x's two alleles / y's two alleles take the observed values
    # under each Jacquard state, by enumerating the IBD partition of
    # (x1, x2, y1, y2) and summing over allele assignments.
    parts = [[0, 0, 0, 0], [0, 0, 1, 1], [0, 0, 0, 1], [0, 0, 1, 2], [0, 1, 0, 0],
             [0, 1, 2, 2], [0, 1, 0, 1], [0, 1, 0, 2], [0, 1, 2, 3]]
    for k, part in enumerate(parts):
        ncls = max(part) + 1
        tot = np.zeros(n)
        for assign in range(1 << ncls):
            al = [(assign >> part[i]) & 1 for i in range(4)]   # 1 = ALT
            ax = al[0] + al[1]
            ay = al[2] + al[3]
            pr = np.ones(n)
            for c in range(ncls):
                pr = pr * np.where((assign >> c) & 1, q, p)
            tot += np.where((gx == ax) & (gy == ay), pr, 0.0)
        L[:, k] = tot
    return L


def fgh(codes_x, codes_y, p, q, keep, delta, eps=1e-8):
    m = (codes_x != 3) & (codes_y != 3) & keep
    L = likelihood_rows(codes_x[m].astype(int), codes_y[m].astype(int), p[m], q[m])
    d = eps + L @ delta
    n = L.shape[0]
    f = -np.sum(np.log(d)) / n
    u = L / d[:, None]
    g = -u.sum(0) / n
    H = u.T @ u / n
    return f, g, H, n
