"""GPU tests of the masked GEMM (matmul_anyway_full_non0tab,
src/impl_matmul_non0tab.rs:163-377) through the C ABI: the reference test's
30 % periodic pattern, masked B entries left NONZERO (the mask alone must
exclude them), transa, ragged blocks, split precision, and the reference's
`unimplemented!` for transb."""
import numpy as np
import pytest

from conftest import check_gemm_summary, load_golden, normwise

pytestmark = pytest.mark.gpu
TOL = 1e-13


def test_matmul_anyway_full_non0tab_golden(cm, wl):
    g = load_golden("matmul_non0tab_pattern30")
    m, n, k, blk = int(g["m"]), int(g["n"]), int(g["k"]), int(g["blksize"])
    a, b, lda, ldb, tab, nblk = wl.ref_matmul_non0tab_inputs(m, n, k, blk)
    c = np.zeros((m, n))
    cm.matmul_anyway_full_non0tab(c, a, b, m, n, k, lda, ldb, n, False, False, tab, nblk)
    check_gemm_summary(c, g, TOL)


@pytest.mark.parametrize("transa", [False, True])
@pytest.mark.parametrize("blk,shape", [(48, (200, 500, 300)), (16, (37, 95, 129)),
                                       (240, (129, 1000, 64))])
def test_non0tab_vs_oracle_nonzero_masked_entries(cm, oracle, transa, blk, shape):
    m, n, k = shape
    rng = np.random.default_rng(m + n + k + blk)
    a = rng.uniform(-1, 1, (k, m) if transa else (m, k))
    b = rng.uniform(-1, 1, (k, n))  # masked entries keep their values
    nblk = -(-n // blk)
    tab = (rng.random((k, nblk)) < 0.3).astype(np.uint8)
    c0 = rng.uniform(-1, 1, (m, n))
    c, ref = c0.copy(), c0.copy()
    cm.MatmulLoops().matmul_loop_parallel_mnk_pack_a_non0tab(c, a, b, m, n, k, a.shape[1], n, n,
                                                             transa, False, tab, nblk, BLKSIZE=blk)
    oracle.matmul_anyway_full_non0tab(ref, a, b, m, n, k, a.shape[1], n, n, transa, False, tab,
                                      nblk, blk)
    assert normwise(c, ref) < TOL


def test_non0tab_any_blksize_vs_dense(cm, wl):
    rng = np.random.default_rng(3)
    m, n, k, blk = 70, 333, 90, 50  # not a multiple of 16: beyond the reference's tiling
    a = rng.uniform(-1, 1, (m, k))
    b = rng.uniform(-1, 1, (k, n))
    nblk = -(-n // blk)
    tab = (rng.random((k, nblk)) < 0.4).astype(np.uint8)
    c = np.zeros((m, n))
    cm.matmul_non0tab_ex(c, a, b, m, n, k, k, n, n, False, False, tab, nblk, blk)
    ref = a @ np.where(wl.expand_mask(tab, n, blk), b, 0.0)
    assert normwise(c, ref) < TOL


def test_non0tab_split_precision(cm, oracle, wl):
    a, b, lda, ldb, tab, nblk = wl.ref_matmul_non0tab_inputs(223, 1000, 223, 48)
    b = b + 0.5  # masked entries nonzero
    c = np.zeros((223, 1000))
    ref = np.zeros((223, 1000))
    cm.matmul_non0tab_ex(c, a, b, 223, 1000, 223, lda, ldb, 1000, False, False, tab, nblk, 48,
                         precision=cm.PREC_OZAKI_INT8)
    oracle.matmul_anyway_full_non0tab(ref, a, b, 223, 1000, 223, lda, ldb, 1000, False, False, tab,
                                      nblk, 48)
    assert normwise(c, ref) < 1e-12


def test_non0tab_transb_is_unimplemented(cm):
    c = np.zeros((4, 48))
    with pytest.raises(NotImplementedError):
        cm.matmul_anyway_full_non0tab(c, np.ones((4, 5)), np.ones((48, 5)), 4, 48, 5, 5, 5, 48,
                                      False, True, np.ones((5, 1), np.uint8), 1)
    assert np.all(c == 0)


def test_non0tab_device_pointers(cm):
    import torch
    m, n, k, blk = 150, 480, 200, 48
    g = torch.Generator(device="cuda").manual_seed(2)
    a = torch.rand(m, k, dtype=torch.float64, device="cuda", generator=g)
    b = torch.rand(k, n, dtype=torch.float64, device="cuda", generator=g)
    tab = (torch.rand(k, n // blk, device="cuda", generator=g) < 0.3).to(torch.uint8)
    c = torch.zeros(m, n, dtype=torch.float64, device="cuda")
    cm.matmul_non0tab_ex(c, a, b, m, n, k, k, n, n, False, False, tab, n // blk, blk)
    torch.cuda.synchronize()
    mask = tab.cpu().numpy().astype(bool).repeat(blk, axis=1)
    ref = a.cpu().numpy() @ np.where(mask, b.cpu().numpy(), 0.0)
    assert normwise(c.cpu().numpy(), ref) < TOL


@pytest.mark.parametrize("prec", [0, 1])
def test_large_masked_host_call_in_blocks(cm, wl, prec):
    """A host-pointer masked GEMM with C above 64 MB runs in blocks of rows
    whose transfers overlap the work: accumulation into a nonzero C, odd
    lda/ldc, the mask whole on the device; (split precision) the same bits as
    one device-pointer call, and within the parity bar of FP64 numpy."""
    import torch
    m, n, k, blk = 1100, 8000, 600, 48
    lda, ldc = k + 5, n + 3
    rng = np.random.default_rng(60 + prec)
    a = rng.uniform(-1, 1, (m, lda))
    b = rng.uniform(-1, 1, (k, n))
    nblk = -(-n // blk)
    tab = (rng.random((k, nblk)) < 0.3).astype(np.uint8)
    c0 = rng.uniform(-1, 1, (m, ldc))
    c = c0.copy()
    cm.matmul_non0tab_ex(c, a, b, m, n, k, lda, n, ldc, False, False, tab, nblk, blk, prec)
    bm = np.where(wl.expand_mask(tab, n, blk), b, 0.0)
    ref = c0[:, :n] + a[:, :k] @ bm
    assert normwise(c[:, :n], ref) < (1e-12 if prec else 1e-13)
    assert np.array_equal(c[:, n:], c0[:, n:])
    if prec:
        dc = torch.from_numpy(c0.copy()).cuda()
        cm.matmul_non0tab_ex(dc, torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda(), m, n, k,
                             lda, n, ldc, False, False, torch.from_numpy(tab).cuda(), nblk, blk,
                             prec)
        torch.cuda.synchronize()
        assert np.array_equal(dc.cpu().numpy(), c)
