"""GPU tests of the split-precision DGEMM (Ozaki scheme on INT8 tcgen05 tensor
cores) through the C ABI.  Bar: within 1e-12 normwise of FP64 (the oracle, or
the reference tests' dense comparator); the reference has no such path, so
the FP64 oracle is the only reference for its accuracy."""
import numpy as np
import pytest

from conftest import check_gemm_summary, load_golden, normwise

pytestmark = pytest.mark.gpu
TOL = 1e-12


def split(cm, c, a, b, m, n, k, lda, ldb, ldc, ta, tb):
    cm.matmul_ex(c, a, b, m, n, k, lda, ldb, ldc, ta, tb, precision=cm.PREC_OZAKI_INT8)


@pytest.mark.parametrize("ta", [False, True])
@pytest.mark.parametrize("tb", [False, True])
@pytest.mark.parametrize("shape", [(1, 1, 1), (7, 300, 33), (129, 257, 128), (200, 300, 500),
                                   (300, 513, 1000)])
def test_split_vs_oracle(cm, oracle, ta, tb, shape):
    m, n, k = shape
    rng = np.random.default_rng(m + 3 * n + 7 * k)
    a = rng.uniform(-1, 1, (k, m) if ta else (m, k))
    b = rng.uniform(-1, 1, (n, k) if tb else (k, n))
    c0 = rng.uniform(-1, 1, (m, n))
    c, ref = c0.copy(), c0.copy()
    split(cm, c, a, b, m, n, k, a.shape[1], b.shape[1], n, ta, tb)
    oracle.matmul_anyway_full(ref, a, b, m, n, k, a.shape[1], b.shape[1], n, ta, tb)
    assert normwise(c, ref) < TOL


@pytest.mark.parametrize("name", ["matmul_nn", "matmul_nt", "matmul_tn", "matmul_tt"])
def test_split_golden(cm, wl, name):
    g = load_golden(name)
    m, n, k, ta, tb = int(g["m"]), int(g["n"]), int(g["k"]), bool(g["transa"]), bool(g["transb"])
    a, b, lda, ldb = wl.ref_matmul_inputs(m, n, k, ta, tb)
    c = np.zeros((m, n))
    split(cm, c, a, b, m, n, k, lda, ldb, n, ta, tb)
    check_gemm_summary(c, g, TOL)


def test_split_wide_dynamic_range(cm, oracle):
    """Rows and columns spanning 2^-300 .. 2^300: the per-row / per-column
    power-of-two scaling must keep each one's own precision."""
    rng = np.random.default_rng(1)
    m, n, k = 64, 80, 96
    a = rng.uniform(-1, 1, (m, k)) * np.ldexp(1.0, rng.integers(-300, 300, m))[:, None]
    b = rng.uniform(-1, 1, (k, n)) * np.ldexp(1.0, rng.integers(-300, 300, n))[None, :]
    c = np.zeros((m, n))
    ref = np.zeros((m, n))
    split(cm, c, a, b, m, n, k, k, n, n, False, False)
    oracle.matmul_anyway_full(ref, a, b, m, n, k, k, n, n, False, False)
    scale = np.abs(a).max(axis=1)[:, None] * np.abs(b).max(axis=0)[None, :] * k
    assert np.max(np.abs(c - ref) / scale) < 1e-14


def test_split_nonfinite_rows_propagate(cm):
    m, n, k = 20, 30, 40
    a = np.ones((m, k))
    b = np.ones((k, n))
    a[3, 5] = np.nan
    b[7, 11] = np.inf
    c = np.zeros((m, n))
    split(cm, c, a, b, m, n, k, k, n, n, False, False)
    assert np.all(np.isnan(c[3, :])) and np.all(np.isnan(c[:, 11]))
    mask = np.ones((m, n), bool)
    mask[3, :] = False
    mask[:, 11] = False
    assert np.allclose(c[mask], k)


def test_split_repeatable(cm, wl):
    a, b, lda, ldb = wl.dgemm_uniform(300, 400, 500, seed=4)
    c1 = np.zeros((300, 400))
    c2 = np.zeros((300, 400))
    split(cm, c1, a, b, 300, 400, 500, lda, ldb, 400, False, False)
    split(cm, c2, a, b, 300, 400, 500, lda, ldb, 400, False, False)
    assert np.array_equal(c1, c2)


def test_split_k_limit(cm):
    c = np.zeros((2, 2))
    a = np.zeros((2, 70000))
    b = np.zeros((70000, 2))
    with pytest.raises(NotImplementedError):
        split(cm, c, a, b, 2, 2, 70000, 70000, 2, 2, False, False)


def test_split_device_pointers(cm):
    import torch
    m, n, k = 257, 300, 700
    g = torch.Generator(device="cuda").manual_seed(3)
    a = torch.rand(m, k, dtype=torch.float64, device="cuda", generator=g) - 0.5
    b = torch.rand(k, n, dtype=torch.float64, device="cuda", generator=g) - 0.5
    c = torch.zeros(m, n, dtype=torch.float64, device="cuda")
    cm.matmul_ex(c, a, b, m, n, k, k, n, n, False, False, precision=cm.PREC_OZAKI_INT8)
    torch.cuda.synchronize()
    assert normwise(c.cpu().numpy(), a.cpu().numpy() @ b.cpu().numpy()) < TOL


@pytest.mark.parametrize("ta,tb", [(False, False), (True, True)])
def test_split_full_size_sampled(cm, wl, ta, tb):
    m, n, k = 3527, 9583, 6581
    a, b, lda, ldb = wl.dgemm_uniform(m, n, k, ta, tb, seed=12)
    c = np.zeros((m, n))
    split(cm, c, a, b, m, n, k, lda, ldb, n, ta, tb)
    rng = np.random.default_rng(5)
    i = rng.integers(0, m, 2048)
    j = rng.integers(0, n, 2048)
    A = a.T if ta else a
    B = b.T if tb else b
    ref = np.einsum("sk,ks->s", A[i, :], B[:, j])
    assert normwise(c[i, j], ref) < TOL


@pytest.mark.parametrize("ta,tb", [(False, False), (True, False), (False, True), (True, True)])
@pytest.mark.parametrize("prec", [0, 1])
def test_large_host_call_in_blocks(cm, ta, tb, prec):
    """A host-pointer call with C above 64 MB runs in blocks of columns whose
    transfers overlap the work: accumulation into a nonzero C, odd lda/ldc, and
    (split precision) the same bits as one device-pointer call."""
    import torch
    m, n, k = 1100, 8000, 600
    lda = (m if ta else k) + 5
    ldc = n + 3
    ldb = (k if tb else n) + 2
    rng = np.random.default_rng(40 + 4 * ta + 2 * tb + prec)
    a = rng.uniform(-1, 1, (k, lda) if ta else (m, lda))
    b = rng.uniform(-1, 1, (n, ldb) if tb else (k, ldb))
    c0 = rng.uniform(-1, 1, (m, ldc))
    c = c0.copy()
    cm.matmul_ex(c, a, b, m, n, k, lda, ldb, ldc, ta, tb, prec)
    A = a[:, :m].T if ta else a[:, :k]
    B = b[:, :k].T if tb else b[:, :n]
    ref = c0[:, :n] + A @ B
    assert normwise(c[:, :n], ref) < (1e-12 if prec else 1e-13)
    assert np.array_equal(c[:, n:], c0[:, n:])  # padding of C untouched
    if prec:
        dc = torch.from_numpy(c0.copy()).cuda()
        cm.matmul_ex(dc, torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda(), m, n, k, lda, ldb,
                     ldc, ta, tb, prec)
        torch.cuda.synchronize()
        assert np.array_equal(dc.cpu().numpy(), c)


@pytest.mark.parametrize("nmod,k", [(14, 33), (15, 1000), (16, 1000), (16, 6581)])
def test_split_moduli_override(cm, oracle, monkeypatch, nmod, k):
    """More moduli than the default (CFGMM_OZAKI_MODULI) scale the operands past
    50 bits, where the residue split takes its 64-bit integer form instead of
    the biased-double form (for A, B or both): same accuracy, to the oracle."""
    monkeypatch.setenv("CFGMM_OZAKI_MODULI", str(nmod))
    m, n = 131, 257
    rng = np.random.default_rng(nmod * 7 + k)
    a = rng.uniform(-1, 1, (m, k))
    b = rng.uniform(-1, 1, (k, n))
    c0 = rng.uniform(-1, 1, (m, n))
    c, ref = c0.copy(), c0.copy()
    split(cm, c, a, b, m, n, k, k, n, n, False, False)
    oracle.matmul_anyway_full(ref, a, b, m, n, k, k, n, n, False, False)
    assert normwise(c, ref) < 1e-13


def test_split_device_call_in_cuda_graph(cm):
    """The device-pointer split call, whose operand preparation forks onto a side
    stream and joins back, records into a CUDA graph: a replay gives the bits of
    a direct call, and a second replay accumulates onto them."""
    import torch
    m, n, k = 257, 300, 700
    g = torch.Generator(device="cuda").manual_seed(8)
    a = torch.rand(m, k, dtype=torch.float64, device="cuda", generator=g) - 0.5
    b = torch.rand(k, n, dtype=torch.float64, device="cuda", generator=g) - 0.5
    ref = torch.zeros(m, n, dtype=torch.float64, device="cuda")
    c = torch.zeros_like(ref)

    def call(out):
        cm.matmul_ex(out, a, b, m, n, k, k, n, n, False, False, precision=cm.PREC_OZAKI_INT8)

    call(ref)
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        call(c)  # warm-up on a side stream before the capture
    torch.cuda.current_stream().wait_stream(s)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        call(c)
    c.zero_()
    graph.replay()
    torch.cuda.synchronize()
    assert torch.equal(c, ref)
    graph.replay()
    torch.cuda.synchronize()
    assert torch.equal(c, 2 * ref)
    del graph
