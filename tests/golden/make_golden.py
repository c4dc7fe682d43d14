"""Generates the golden fixtures in this directory.

The reference (Rust) cannot be built or run in this image, and its tests hold
no golden values: each one prints the max error of the reference against a
dense FP64 evaluation by OpenBLAS (rstsr) and asserts nothing
(src/impl_matmul.rs:297-397, src/impl_matmul_non0tab.rs:328-377,
src/impl_aodmao2rho.rs:263-425).  These fixtures therefore hold that
comparator's values -- dense FP64 by numpy's OpenBLAS -- on the reference
tests' own input generators (sin / cos flat-index inputs, the 25 % and 30 %
periodic non0tab patterns, masked phi zeroed), at sizes that run in seconds.
Inputs are regenerated by the tests from the recorded parameters; only
outputs (or, for GEMMs, row sums, column sums and seeded sampled entries) are
stored.

Usage: python tests/golden/make_golden.py
"""
from __future__ import annotations

import importlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
wl = importlib.import_module("cfgable-matmul_b200.workloads")

GEMM_CASES = {  # name: (m, n, k, transa, transb)
    "matmul_nn": (357, 958, 658, False, False),
    "matmul_nt": (357, 958, 658, False, True),
    "matmul_tn": (357, 958, 658, True, False),
    "matmul_tt": (357, 958, 658, True, True),
}
AODM_CASES = {  # name: (nao, ngrid, nset, blksize, dense)
    "aodmao2rho_pattern25": (300, 1025, 1, 48, False),
    "aodmao2rho_all_dense": (300, 1025, 1, 48, True),
    "aodmao2rho_pattern25_nset2_blk64": (211, 777, 2, 64, False),
}
NON0TAB_CASES = {  # name: (m, n, k, blksize)
    "matmul_non0tab_pattern30": (223, 1000, 223, 48),
}
NSAMPLE = 4096


def sample_idx(m, n, seed=1234):
    rng = np.random.default_rng(seed)
    return rng.integers(0, m, NSAMPLE), rng.integers(0, n, NSAMPLE)


def gemm_summary(c):
    i, j = sample_idx(*c.shape)
    return dict(row_sums=c.sum(axis=1), col_sums=c.sum(axis=0), sample_i=i, sample_j=j,
                sample=c[i, j], absmax=np.abs(c).max())


def main():
    for name, (m, n, k, ta, tb) in GEMM_CASES.items():
        a, b, lda, ldb = wl.ref_matmul_inputs(m, n, k, ta, tb)
        c = (a.T if ta else a) @ (b.T if tb else b)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), m=m, n=n, k=k, transa=ta,
                            transb=tb, **gemm_summary(c))
    for name, (nao, ngrid, nset, blk, dense) in AODM_CASES.items():
        lhs, rhs, dm, tab, nblk = wl.ref_aodmao2rho_inputs(nao, ngrid, nset, blk, dense)
        rho = wl.dense_rho(lhs, rhs, dm, tab, blk)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), nao=nao, ngrid=ngrid, nset=nset,
                            blksize=blk, dense=dense, rho=rho)
    for name, (m, n, k, blk) in NON0TAB_CASES.items():
        a, b, lda, ldb, tab, nblk = wl.ref_matmul_non0tab_inputs(m, n, k, blk)
        c = a @ b  # masked B entries are zero, as in the reference test
        np.savez_compressed(os.path.join(HERE, name + ".npz"), m=m, n=n, k=k, blksize=blk,
                            **gemm_summary(c))
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main()
