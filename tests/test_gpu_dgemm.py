"""GPU parity tests of the FP64 DGEMM through the C ABI.

Named after the reference's own tests (src/impl_matmul.rs:297-397) and using
their generators; unlike the reference they assert a tolerance: FP64 results
within 1e-13 normwise (max|C - C_ref| / max|C_ref|) of the oracle or of the
reference tests' dense comparator.  The reference has no TT test; one is added.
"""
import numpy as np
import pytest

from conftest import check_gemm_summary, load_golden, normwise

pytestmark = pytest.mark.gpu
TOL = 1e-13


@pytest.mark.parametrize("name", ["matmul_nn", "matmul_nt", "matmul_tn", "matmul_tt"])
def test_matmul_golden(cm, wl, name):
    g = load_golden(name)
    m, n, k, ta, tb = int(g["m"]), int(g["n"]), int(g["k"]), bool(g["transa"]), bool(g["transb"])
    a, b, lda, ldb = wl.ref_matmul_inputs(m, n, k, ta, tb)
    c = np.zeros((m, n))
    cm.matmul_anyway_full(c, a, b, m, n, k, lda, ldb, n, ta, tb)
    check_gemm_summary(c, g, TOL)


@pytest.mark.parametrize("ta", [False, True])
@pytest.mark.parametrize("tb", [False, True])
@pytest.mark.parametrize("shape", [(1, 1, 1), (1, 300, 7), (129, 1, 33), (127, 255, 17),
                                   (256, 384, 512), (333, 257, 1000)])
def test_matmul_vs_oracle(cm, oracle, ta, tb, shape):
    m, n, k = shape
    rng = np.random.default_rng(m * 7 + n * 3 + k)
    a = rng.uniform(-1, 1, (k, m) if ta else (m, k))
    b = rng.uniform(-1, 1, (n, k) if tb else (k, n))
    c0 = rng.uniform(-1, 1, (m, n))  # accumulate into a nonzero C
    c, cref = c0.copy(), c0.copy()
    cm.matmul_anyway_full(c, a, b, m, n, k, a.shape[1], b.shape[1], n, ta, tb)
    oracle.matmul_anyway_full(cref, a, b, m, n, k, a.shape[1], b.shape[1], n, ta, tb)
    assert normwise(c, cref) < TOL


@pytest.mark.parametrize("ta,tb", [(False, False), (True, True)])
def test_matmul_padded_and_odd_ld(cm, oracle, ta, tb):
    """ld larger than the row length (odd, so rows start 8 bytes off 16-byte
    alignment), and a C with padding columns that must stay untouched."""
    m, n, k = 150, 170, 190
    lda, ldb, ldc = (m if ta else k) + 13, (k if tb else n) + 7, n + 5
    rng = np.random.default_rng(5)
    a = rng.uniform(-1, 1, ((k if ta else m), lda))
    b = rng.uniform(-1, 1, ((n if tb else k), ldb))
    c = rng.uniform(-1, 1, (m, ldc))
    cref = c.copy()
    cm.matmul_anyway_full(c, a, b, m, n, k, lda, ldb, ldc, ta, tb)
    oracle.matmul_anyway_full(cref, a, b, m, n, k, lda, ldb, ldc, ta, tb)
    assert normwise(c, cref) < TOL
    assert np.array_equal(c[:, n:], cref[:, n:])


def test_matmul_aliases_and_struct(cm, wl):
    m, n, k = 100, 90, 80
    a, b, lda, ldb = wl.ref_matmul_inputs(m, n, k)
    ref = a @ b
    loops = cm.MatmulLoops(np.float64, 252, 512, 240, 14, 2, 8)
    for f in (loops.matmul_loop_parallel_mnk_pack_a, loops.matmul_loop_macro_mb,
              cm.matmul_anyway_full):
        c = np.zeros((m, n))
        f(c, a, b, m, n, k, lda, ldb, n, False, False)
        assert normwise(c, ref) < TOL


def test_matmul_device_pointers(cm):
    import torch
    m, n, k = 300, 200, 100
    g = torch.Generator(device="cuda").manual_seed(0)
    a = torch.rand(m, k, dtype=torch.float64, device="cuda", generator=g)
    b = torch.rand(k, n, dtype=torch.float64, device="cuda", generator=g)
    c = torch.ones(m, n, dtype=torch.float64, device="cuda")
    cm.matmul_anyway_full(c, a, b, m, n, k, k, n, n, False, False)
    torch.cuda.synchronize()
    ref = 1.0 + a.cpu().numpy() @ b.cpu().numpy()
    assert normwise(c.cpu().numpy(), ref) < TOL


def test_matmul_repeatable(cm, wl):
    """The GPU sum order is fixed per element: two calls agree bit for bit."""
    a, b, lda, ldb = wl.dgemm_uniform(500, 600, 700, seed=2)
    c1 = np.zeros((500, 600))
    c2 = np.zeros((500, 600))
    cm.matmul_anyway_full(c1, a, b, 500, 600, 700, lda, ldb, 600, False, False)
    cm.matmul_anyway_full(c2, a, b, 500, 600, 700, lda, ldb, 600, False, False)
    assert np.array_equal(c1, c2)


@pytest.mark.parametrize("ta,tb", [(False, False), (False, True), (True, False), (True, True)])
def test_matmul_full_size_sampled(cm, wl, ta, tb):
    """The 3527x6581 by 6581x9583 workload: 2048 seeded entries checked
    against FP64 dot products (a size-independent check)."""
    m, n, k = 3527, 9583, 6581
    a, b, lda, ldb = wl.dgemm_uniform(m, n, k, ta, tb, seed=11)
    c = np.zeros((m, n))
    cm.matmul_anyway_full(c, a, b, m, n, k, lda, ldb, n, ta, tb)
    rng = np.random.default_rng(3)
    i = rng.integers(0, m, 2048)
    j = rng.integers(0, n, 2048)
    A = a.T if ta else a
    B = b.T if tb else b
    ref = np.einsum("sk,ks->s", A[i, :], B[:, j])
    assert normwise(c[i, j], ref) < TOL
