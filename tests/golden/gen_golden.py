"""Generates tests/golden/block_multiply_golden.npz from TAMM's OWN compiled block
kernels (oracle/_ref/libtamm_ref.so, built from the TAMM sources by oracle/Makefile).

    python tests/golden/gen_golden.py

Inputs are regenerated from seeds by the oracle's counter-based generator, so only
outputs are stored.  Needs oracle/_ref (i.e. the TAMM source tree at build time).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, os.path.dirname(HERE))

from oracle import oracle as O  # noqa: E402
import test_oracle as T  # noqa: E402


def main():
    assert O.ref() is not None, "oracle/_ref/libtamm_ref.so is required"
    out = {}
    for idx, (cl, al, bl) in enumerate(T.PATTERNS):
        for beta in (1.0, 0.0, 0.5):
            for is_assign in (0, 1):
                A, B, C0 = T._mk(al, 1), T._mk(bl, 2), T._mk(cl, 3)
                C = np.array(C0, copy=True)
                rc = O.block_multiply(1.3, A, [T.LAB[c] for c in al], B, [T.LAB[c] for c in bl], beta,
                                      C, [T.LAB[c] for c in cl], is_assign, "ref")
                assert rc == 0
                out[f"p{idx}_b{beta}_a{is_assign}"] = C.reshape(-1)
    A = np.zeros((10, 10, 10, 10))
    B = np.zeros((10, 10, 10, 10))
    O.fill_uniform(A.reshape(-1), 0, 0)
    O.fill_uniform(B.reshape(-1), 0, A.size)
    C = np.zeros((10, 10, 10, 10))
    lab = {c: -ord(c) for c in "abcijk"}
    assert O.block_multiply(1.0, A, [lab[c] for c in "acik"], B, [lab[c] for c in "cbkj"], 1.0, C,
                            [lab[c] for c in "abij"], 0, "ref") == 0
    out["config1_block"] = C.reshape(-1)
    lad = T.small_ladder("ref")
    out["ladder_r2"] = lad.data[:lad.total].copy()
    np.savez_compressed(os.path.join(HERE, "block_multiply_golden.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main()
