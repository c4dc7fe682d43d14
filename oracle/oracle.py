"""ctypes front end of the CPU oracle (oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()``
as the checker and by ``bench.py`` for its CPU-baseline leg.  The product
(the ``cfgable-matmul_b200`` package and ``libcfgmm.so``) never imports it.

PARITY UNPINNED: the reference is Rust and cannot be built or run in this
image, and its tests hold no golden values.  The restatement is checked against
the reference tests' own comparator (dense FP64 with OpenBLAS, here numpy) on
the reference tests' own generators; see tests/golden/.

All arrays are numpy float64 / uint8 and are used in place (outputs are
accumulated into, as in the reference: impl_matmul.rs:31-46,
impl_aodmao2rho.rs:77-92).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None


def _has_avx512() -> bool:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    return "avx512f" in line.split()
    except OSError:
        pass
    return False


def build(force: bool = False) -> None:
    """Compiles both ISA variants of the oracle with its Makefile."""
    targets = [os.path.join(_HERE, n) for n in ("liboracle_v3.so", "liboracle_v4.so")]
    if force or not all(os.path.exists(t) for t in targets):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        name = "liboracle_v4.so" if _has_avx512() else "liboracle_v3.so"
        path = os.path.join(_HERE, name)
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        P, S, I = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int
        L.oracle_matmul_anyway_full.argtypes = [P, P, P] + [S] * 6 + [I, I, I]
        L.oracle_matmul_anyway_full.restype = I
        L.oracle_matmul_anyway_full_non0tab.argtypes = [P, P, P] + [S] * 6 + [I, I, P, S, S, I]
        L.oracle_matmul_anyway_full_non0tab.restype = I
        L.oracle_aodmao2rho.argtypes = [P, P, P, P] + [S] * 5 + [P, S, S, I]
        L.oracle_aodmao2rho.restype = I
        L.oracle_aodm_fock.argtypes = [P, P, P, P] + [S] * 5 + [P, S, S, I]
        L.oracle_aodm_fock.restype = I
        L.oracle_max_threads.restype = I
        _lib = L
    return _lib


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def _check(a: np.ndarray, dtype) -> None:
    if a.dtype != dtype or not a.flags.c_contiguous:
        raise TypeError(f"expected a C-contiguous {np.dtype(dtype).name} array")


def max_threads() -> int:
    return lib().oracle_max_threads()


def matmul_anyway_full(c, a, b, m, n, k, lda, ldb, ldc, transa, transb, nthreads=0) -> None:
    """C += op(A) op(B) by the restated matmul_loop_parallel_mnk_pack_a
    (impl_matmul.rs:155-231) with the matmul_anyway_full tuning
    (impl_matmul.rs:234-248)."""
    for x in (c, a, b):
        _check(x, np.float64)
    rc = lib().oracle_matmul_anyway_full(_ptr(c), _ptr(a), _ptr(b), m, n, k, lda, ldb, ldc,
                                         int(transa), int(transb), nthreads)
    if rc != 0:
        raise ValueError(f"oracle_matmul_anyway_full returned {rc}")


def matmul_anyway_full_non0tab(c, a, b, m, n, k, lda, ldb, ldc, transa, transb, tab, ldtab,
                               blksize=48, nthreads=0) -> None:
    """C[i,j] += sum_{p: tab[p, j/BLK]} op(A)[i,p] B[p,j]
    (impl_matmul_non0tab.rs:210-326).  transb raises, as the reference panics."""
    for x in (c, a, b):
        _check(x, np.float64)
    _check(tab, np.uint8)
    rc = lib().oracle_matmul_anyway_full_non0tab(_ptr(c), _ptr(a), _ptr(b), m, n, k, lda, ldb,
                                                 ldc, int(transa), int(transb), _ptr(tab), ldtab,
                                                 blksize, nthreads)
    if rc == -2:
        raise NotImplementedError("transb=true is not implemented for the masked GEMM")
    if rc != 0:
        raise ValueError(f"oracle_matmul_anyway_full_non0tab returned {rc}")


def aodmao2rho(rhos, dms, ao_lhs, ao_rhs, strides, shape, nset, tab, ldtab, blksize=48,
               nthreads=0) -> None:
    """rho[s,g] += sum_{u,v active in g's block} ao_lhs[u,g] D_s[u,v] ao_rhs[v,g]
    by the restated aodmao2rho_loop_parallel (impl_aodmao2rho.rs:171-244)."""
    for x in (rhos, dms, ao_lhs, ao_rhs):
        _check(x, np.float64)
    _check(tab, np.uint8)
    stride_ao, stride_grid = strides
    nao, ngrid = shape
    rc = lib().oracle_aodmao2rho(_ptr(rhos), _ptr(dms), _ptr(ao_lhs), _ptr(ao_rhs), stride_ao,
                                 stride_grid, nao, ngrid, nset, _ptr(tab), ldtab, blksize,
                                 nthreads)
    if rc != 0:
        raise ValueError(f"oracle_aodmao2rho returned {rc}")


def aodm_fock(vs, ws, ao_lhs, ao_rhs, strides, shape, nset, tab, ldtab, blksize=48,
              nthreads=0) -> None:
    """V_s[u,v] += sum over g in blocks where u and v are both active of
    ao_lhs[u,g] w_s[g] ao_rhs[v,g]: the transpose of aodmao2rho on the same
    layouts and mask, written from that formula."""
    for x in (vs, ws, ao_lhs, ao_rhs):
        _check(x, np.float64)
    _check(tab, np.uint8)
    stride_ao, stride_grid = strides
    nao, ngrid = shape
    rc = lib().oracle_aodm_fock(_ptr(vs), _ptr(ws), _ptr(ao_lhs), _ptr(ao_rhs), stride_ao,
                                stride_grid, nao, ngrid, nset, _ptr(tab), ldtab, blksize,
                                nthreads)
    if rc != 0:
        raise ValueError(f"oracle_aodm_fock returned {rc}")
