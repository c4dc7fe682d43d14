"""GPU tests of the packed, TMA-staged form of the FP64 DGEMM (products of
2e9 flops and more): every transpose, odd and padded leading dimensions,
accumulation into a nonzero C, the K split of a last partial wave of tiles,
and the masked GEMM whose mask is applied while packing.  FP64 results within
1e-13 normwise of numpy's FP64 product."""
import numpy as np
import pytest

from conftest import normwise

pytestmark = pytest.mark.gpu
TOL = 1e-13


def _op(x, t):
    return x.T if t else x


@pytest.mark.parametrize("transa,transb", [(False, False), (False, True), (True, False),
                                           (True, True)])
@pytest.mark.parametrize("m,n,k,pad", [(1000, 1200, 1100, 0), (2000, 1500, 701, 3),
                                       (1037, 1161, 1999, 1)])
def test_packed_dgemm(cm, transa, transb, m, n, k, pad):
    rng = np.random.default_rng(m + n + k + 2 * transa + transb)
    ar, ac = (k, m) if transa else (m, k)
    br, bc = (n, k) if transb else (k, n)
    lda, ldb, ldc = ac + pad, bc + 2 * pad, n + pad
    a = rng.uniform(-1, 1, (ar, lda))
    b = rng.uniform(-1, 1, (br, ldb))
    c = rng.uniform(-1, 1, (m, ldc))
    ref = c.copy()
    ref[:, :n] += _op(a[:, :ac], transa) @ _op(b[:, :bc], transb)
    cm.matmul_anyway_full(c, a, b, m, n, k, lda, ldb, ldc, transa, transb)
    assert normwise(c[:, :n], ref[:, :n]) < TOL
    assert np.array_equal(c[:, n:], ref[:, n:])  # padding untouched


@pytest.mark.parametrize("transa", [False, True])
def test_packed_masked_gemm(cm, wl, transa):
    m, n, k, blk = 1100, 1300, 1500, 48
    rng = np.random.default_rng(11 + transa)
    a = rng.uniform(-1, 1, (k, m) if transa else (m, k))
    b = rng.uniform(-1, 1, (k, n))  # masked entries hold nonzero values
    nblk = -(-n // blk)
    tab = (rng.random((k, nblk)) < 0.3).astype(np.uint8)
    c = np.zeros((m, n))
    cm.matmul_non0tab_ex(c, a, b, m, n, k, a.shape[1], n, n, transa, False, tab, nblk, blk)
    bm = np.where(wl.expand_mask(tab, n, blk), b, 0.0)
    ref = _op(a, transa) @ bm
    assert normwise(c, ref) < TOL


def test_packed_matches_unpacked_within_tolerance(cm, monkeypatch):
    """The same product through both forms (the packed one on by size)."""
    import subprocess, sys, os, json
    code = ("import importlib,sys,numpy as np; sys.path.insert(0,'.');"
            "cm=importlib.import_module('cfgable-matmul_b200');"
            "r=np.random.default_rng(3); a=r.uniform(-1,1,(1300,1201)); b=r.uniform(-1,1,(1201,1400));"
            "c=np.zeros((1300,1400)); cm.matmul_anyway_full(c,a,b,1300,1400,1201,1201,1400,1400,False,False);"
            "np.save(sys.argv[1], c)")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    outs = []
    for thr in ("1e9", "-1"):
        path = os.path.join(os.environ.get("TMPDIR", "/tmp"), f"cfgmm_pack_{thr}.npy")
        env = dict(os.environ, CFGMM_DGEMM_PACK_MIN_FLOPS=thr)
        subprocess.run([sys.executable, "-c", code, path], cwd=root, env=env, check=True)
        outs.append(np.load(path))
    assert normwise(outs[0], outs[1]) < 1e-14
