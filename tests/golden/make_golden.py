"""Writes tests/golden/config0_oracle.npz: the config-0 cohort (N=64 x M=10,000,
seeded synthetic genotypes) and the FP64 oracle's rows for all of its pairs.

The reference (Rust) cannot be built here, so these rows are the oracle's own,
kept as a regression anchor: the CPU tests check that the oracle still
reproduces them, and the GPU tests compare the CUDA path against them.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def main():
    from kestrel_b200 import synth
    from oracle import pyoracle
    pyoracle.build()
    c = synth.config0()
    rows = pyoracle.relatedness(c.codes)
    np.savez_compressed(os.path.join(HERE, "config0_oracle.npz"), codes=c.codes,
                        x=rows["x"], y=rows["y"], jacquard=rows["jacquard"], obj=rows["obj"],
                        iters=rows["iters"], cond=rows["cond"])
    print(f"{len(rows)} rows written")


if __name__ == "__main__":
    main()
