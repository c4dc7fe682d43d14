"""CPU tests of the oracle (the C++ restatement of the reference's loops).

The reference cannot run here (Rust, no toolchain), and its tests carry no
golden values, so the oracle is pinned against the comparator the reference's
tests print their "Max error" against -- dense FP64 (OpenBLAS) -- on the
reference tests' own generators (tests/golden/), and against plain-Python
loop restatements of the per-block compaction on tiny inputs.
"""
import numpy as np
import pytest

from conftest import check_gemm_summary, load_golden as _load, normwise

TOL = 1e-13


@pytest.mark.parametrize("name", ["matmul_nn", "matmul_nt", "matmul_tn", "matmul_tt"])
@pytest.mark.parametrize("nthreads", [1, 0])
def test_oracle_matmul_golden(oracle, wl, name, nthreads):
    g = _load(name)
    m, n, k, ta, tb = int(g["m"]), int(g["n"]), int(g["k"]), bool(g["transa"]), bool(g["transb"])
    a, b, lda, ldb = wl.ref_matmul_inputs(m, n, k, ta, tb)
    c = np.zeros((m, n))
    oracle.matmul_anyway_full(c, a, b, m, n, k, lda, ldb, n, ta, tb, nthreads=nthreads)
    check_gemm_summary(c, g, TOL)


@pytest.mark.parametrize("name", ["aodmao2rho_pattern25", "aodmao2rho_all_dense",
                                  "aodmao2rho_pattern25_nset2_blk64"])
@pytest.mark.parametrize("nthreads", [1, 0])
def test_oracle_aodmao2rho_golden(oracle, wl, name, nthreads):
    g = _load(name)
    nao, ngrid, nset, blk = int(g["nao"]), int(g["ngrid"]), int(g["nset"]), int(g["blksize"])
    lhs, rhs, dm, tab, nblk = wl.ref_aodmao2rho_inputs(nao, ngrid, nset, blk, bool(g["dense"]))
    rho = np.zeros((nset, ngrid))
    oracle.aodmao2rho(rho, dm, lhs, rhs, (nao, ngrid), (nao, ngrid), nset, tab, nblk, blk,
                      nthreads=nthreads)
    assert normwise(rho, g["rho"]) < TOL


def test_oracle_matmul_non0tab_golden(oracle, wl):
    g = _load("matmul_non0tab_pattern30")
    m, n, k, blk = int(g["m"]), int(g["n"]), int(g["k"]), int(g["blksize"])
    a, b, lda, ldb, tab, nblk = wl.ref_matmul_non0tab_inputs(m, n, k, blk)
    c = np.zeros((m, n))
    oracle.matmul_anyway_full_non0tab(c, a, b, m, n, k, lda, ldb, n, False, False, tab, nblk, blk)
    check_gemm_summary(c, g, TOL)


def test_oracle_non0tab_transb_panics(oracle, wl):
    a, b, lda, ldb, tab, nblk = wl.ref_matmul_non0tab_inputs(16, 48, 16, 48)
    c = np.zeros((16, 48))
    with pytest.raises(NotImplementedError):
        oracle.matmul_anyway_full_non0tab(c, a, b, 16, 48, 16, lda, ldb, 48, False, True, tab, nblk)


def _python_rho(lhs, rhs, dms, tab, blk):
    """Plain-Python restatement: per block, the active list by the reference's
    get_indices_from_non0tab (impl_matmul_non0tab.rs:118-129), skip when empty
    (impl_aodmao2rho.rs:130-132), then the double sum over the list."""
    nao, ngrid = lhs.shape
    rho = np.zeros((len(dms), ngrid))
    for g in range(ngrid):
        b = g // blk
        idx = [p for p in range(nao) if tab[p, b]]
        if not idx:
            continue
        for s, d in enumerate(dms):
            tot = 0.0
            for u in idx:
                x = 0.0
                for v in idx:
                    x += d[u, v] * rhs[v, g]
                tot += x * lhs[u, g]
            rho[s, g] += tot
    return rho


@pytest.mark.parametrize("blk", [16, 32, 48])
def test_oracle_matches_python_loops(oracle, blk):
    rng = np.random.default_rng(blk)
    nao, ngrid, nset = 23, 77, 2
    nblk = -(-ngrid // blk)
    lhs = rng.standard_normal((nao, ngrid))
    rhs = rng.standard_normal((nao, ngrid))  # NOT zeroed in masked tiles:
    dms = rng.uniform(-1, 1, (nset, nao, nao))  # the mask alone must exclude them
    tab = (rng.random((nao, nblk)) < 0.4).astype(np.uint8)
    tab[:, 0] = 0  # one fully masked block
    rho = np.zeros((nset, ngrid))
    oracle.aodmao2rho(rho, dms, lhs, rhs, (nao, ngrid), (nao, ngrid), nset, tab, nblk, blk,
                      nthreads=1)
    ref = _python_rho(lhs, rhs, dms, tab, blk)
    assert normwise(rho, ref) < 1e-14
    assert np.all(rho[:, :blk] == 0.0)


def test_oracle_threads_agree(oracle, wl):
    p = wl.small_masked(seed=3, nao=256, ngrid=2048, nset=2)
    r1 = np.zeros((p.nset, p.ngrid))
    r8 = np.zeros((p.nset, p.ngrid))
    for r, nt in ((r1, 1), (r8, 0)):
        oracle.aodmao2rho(r, p.dms, p.ao, p.ao, (p.nao, p.ngrid), (p.nao, p.ngrid), p.nset, p.tab,
                          p.nblk, p.blksize, nthreads=nt)
    assert normwise(r8, r1) < 1e-14
    assert normwise(r1, wl.dense_rho(p.ao, p.ao, p.dms, p.tab, p.blksize)) < TOL


def test_oracle_accumulates(oracle, wl):
    a, b, lda, ldb = wl.ref_matmul_inputs(30, 40, 50)
    c0 = np.arange(30 * 40, dtype=np.float64).reshape(30, 40)
    c = c0.copy()
    oracle.matmul_anyway_full(c, a, b, 30, 40, 50, lda, ldb, 40, False, False)
    assert normwise(c, c0 + a @ b) < TOL


def test_generators_shapes(wl):
    p = wl.geometric(seed=1, nao=120, nshell=24, natom=8, ngrid=640, nset=2)
    assert p.ao.shape == (120, 640) and p.tab.shape == (120, 10) and p.dms.shape == (2, 120, 120)
    assert int(p.shell_sizes.sum()) == 120
    assert set(np.unique(p.shell_sizes)) <= {1, 3, 5, 7}
    assert np.allclose(p.dms, p.dms.transpose(0, 2, 1))
    mask = wl.expand_mask(p.tab, p.ngrid, p.blksize)
    assert np.all(p.ao[~mask] == 0.0)
    assert abs(p.tab.astype(float).mean() - 0.3) < 0.1


def _python_fock(lhs, rhs, ws, tab, blk):
    """V_s[u,v] = sum over g with u and v active in g's block of lhs[u,g] w_s[g] rhs[v,g]."""
    nao, ngrid = lhs.shape
    vs = np.zeros((ws.shape[0], nao, nao))
    for s in range(ws.shape[0]):
        for g in range(ngrid):
            idx = [u for u in range(nao) if tab[u, g // blk]]
            for u in idx:
                for v in idx:
                    vs[s, u, v] += lhs[u, g] * ws[s, g] * rhs[v, g]
    return vs


@pytest.mark.parametrize("blk", [16, 48, 100])
def test_oracle_fock_matches_python_loops(oracle, blk):
    rng = np.random.default_rng(100 + blk)
    nao, ngrid, nset = 19, 203, 2
    nblk = -(-ngrid // blk)
    lhs = rng.standard_normal((nao, ngrid))
    rhs = rng.standard_normal((nao, ngrid))  # nonzero where masked: the mask must exclude them
    ws = rng.uniform(0, 1, (nset, ngrid))
    tab = (rng.random((nao, nblk)) < 0.5).astype(np.uint8)
    tab[:, -1] = 0
    vs = np.zeros((nset, nao, nao))
    oracle.aodm_fock(vs, ws, lhs, rhs, (nao, ngrid), (nao, ngrid), nset, tab, nblk, blk)
    assert normwise(vs, _python_fock(lhs, rhs, ws, tab, blk)) < 1e-14


def test_oracle_fock_is_the_adjoint_of_aodmao2rho(oracle, wl):
    """sum_uv V(w)[u,v] D[u,v] == sum_g w[g] rho(D)[g] on the same phi and mask."""
    p = wl.small_masked(seed=5, nao=96, ngrid=960, nset=1)
    rng = np.random.default_rng(5)
    w = rng.uniform(0, 1, (1, p.ngrid))
    rho = np.zeros((1, p.ngrid))
    oracle.aodmao2rho(rho, p.dms, p.ao, p.ao, (p.nao, p.ngrid), (p.nao, p.ngrid), 1, p.tab,
                      p.nblk, p.blksize)
    v = np.zeros((1, p.nao, p.nao))
    oracle.aodm_fock(v, w, p.ao, p.ao, (p.nao, p.ngrid), (p.nao, p.ngrid), 1, p.tab, p.nblk,
                     p.blksize)
    lhs, rhs = float(np.sum(v * p.dms)), float(np.sum(w * rho))
    assert abs(lhs - rhs) <= 1e-12 * max(1.0, abs(rhs))


def test_oracle_fock_threads_bitwise(oracle, wl):
    p = wl.small_masked(seed=6, nao=136, ngrid=700, nset=2)
    ws = np.random.default_rng(6).uniform(0, 1, (p.nset, p.ngrid))
    v1 = np.ones((p.nset, p.nao + 3, p.nao + 3))  # padded rows, accumulated into
    v8 = v1.copy()
    for v, nt in ((v1, 1), (v8, 0)):
        oracle.aodm_fock(v, ws, p.ao, p.ao, (p.nao + 3, p.ngrid), (p.nao, p.ngrid), p.nset,
                         p.tab, p.nblk, p.blksize, nthreads=nt)
    assert np.array_equal(v1, v8)
    assert np.all(v1[:, p.nao:, :] == 1.0) and np.all(v1[:, :, p.nao:] == 1.0)
