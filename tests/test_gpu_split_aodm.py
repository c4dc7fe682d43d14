"""GPU tests of the split-precision masked AO-DM-AO contraction (slice-form
Ozaki scheme on INT8 tcgen05 tensor cores) through the C ABI.  Bar: within
1e-12 normwise of the FP64 oracle, with the reference's semantics (masked
entries excluded whatever phi holds there, empty blocks untouched)."""
import numpy as np
import pytest

from conftest import load_golden, normwise

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.fixture(autouse=True, params=["row", "pair"])
def split_form(request, monkeypatch):
    """Every test runs both forms of the split kernel: the row form (one
    block tile per item) and the pair form (two paired block tiles per item,
    the default from 1024 AOs and 8192 points on)."""
    monkeypatch.setenv("CFGMM_SPLIT_FORM", request.param)
    return request.param


def split(cm, rho, dms, lhs, rhs, strides, shape, nset, tab, ldtab, blk):
    cm.aodmao2rho_ex(rho, dms, lhs, rhs, strides, shape, nset, tab, ldtab, blk,
                     precision=cm.PREC_OZAKI_INT8)


@pytest.mark.parametrize("name", ["aodmao2rho_pattern25", "aodmao2rho_all_dense",
                                  "aodmao2rho_pattern25_nset2_blk64"])
def test_split_aodm_golden(cm, wl, name):
    g = load_golden(name)
    nao, ngrid, nset, blk = int(g["nao"]), int(g["ngrid"]), int(g["nset"]), int(g["blksize"])
    lhs, rhs, dm, tab, nblk = wl.ref_aodmao2rho_inputs(nao, ngrid, nset, blk, bool(g["dense"]))
    rho = np.zeros((nset, ngrid))
    split(cm, rho, dm, lhs, rhs, (nao, ngrid), (nao, ngrid), nset, tab, nblk, blk)
    assert normwise(rho, g["rho"]) < TOL


@pytest.mark.parametrize("maker", ["small", "geometric"])
def test_split_aodm_workloads(cm, oracle, wl, maker):
    p = wl.small_masked(seed=0) if maker == "small" else wl.geometric(seed=0)
    rho = np.zeros((p.nset, p.ngrid))
    ref = np.zeros((p.nset, p.ngrid))
    args = ((p.nao, p.ngrid), (p.nao, p.ngrid), p.nset, p.tab, p.nblk, p.blksize)
    split(cm, rho, p.dms, p.ao, p.ao, *args)
    oracle.aodmao2rho(ref, p.dms, p.ao, p.ao, *args)
    assert normwise(rho, ref) < TOL


@pytest.mark.parametrize("blk", [16, 48, 64, 100, 200])
@pytest.mark.parametrize("nset", [1, 3, 4])
def test_split_aodm_ragged_sets_masked_entries(cm, wl, blk, nset):
    rng = np.random.default_rng(blk + 10 * nset)
    nao, ngrid = 301, 1111
    nblk = -(-ngrid // blk)
    lhs = rng.standard_normal((nao, ngrid))
    rhs = rng.standard_normal((nao, ngrid))  # masked entries stay nonzero on purpose
    dms = rng.uniform(-1, 1, (nset, nao, nao))  # not symmetric
    tab = (rng.random((nao, nblk)) < 0.3).astype(np.uint8)
    tab[:, 1] = 0  # an empty block
    rho0 = rng.standard_normal((nset, ngrid))
    rho = rho0.copy()
    split(cm, rho, dms, lhs, rhs, (nao, ngrid), (nao, ngrid), nset, tab, nblk, blk)
    ref = rho0 + wl.dense_rho(lhs, rhs, dms, tab, blk)
    assert normwise(rho - rho0, ref - rho0) < TOL
    g0, g1 = blk, min(2 * blk, ngrid)
    assert np.array_equal(rho[:, g0:g1], rho0[:, g0:g1])


def test_split_aodm_wide_range_and_nonfinite(cm, wl):
    rng = np.random.default_rng(5)
    nao, ngrid, blk = 96, 640, 64
    nblk = ngrid // blk
    ao = rng.standard_normal((nao, ngrid)) * np.ldexp(1.0, rng.integers(-200, 200, ngrid))[None, :]
    dms = rng.uniform(-1, 1, (1, nao, nao)) * np.ldexp(1.0, rng.integers(-200, 200, nao))[None, :, None]
    tab = np.ones((nao, nblk), np.uint8)
    rho = np.zeros((1, ngrid))
    split(cm, rho, dms, ao, ao, (nao, ngrid), (nao, ngrid), 1, tab, nblk, blk)
    ref = wl.dense_rho(ao, ao, dms, tab, blk)
    bound = wl.dense_rho(np.abs(ao), np.abs(ao), np.abs(dms), tab, blk)
    assert np.max(np.abs(rho - ref) / bound) < 1e-13  # relative to sum |phi||D||phi|
    dms[0, 5, 7] = np.nan
    rho = np.zeros((1, ngrid))
    split(cm, rho, dms, ao, ao, (nao, ngrid), (nao, ngrid), 1, tab, nblk, blk)
    assert np.all(np.isnan(rho))


def test_split_aodm_device_pointers_repeatable(cm, wl):
    import torch
    p = wl.small_masked(seed=6, nset=2)
    ao = torch.from_numpy(p.ao).cuda()
    dms = torch.from_numpy(p.dms).cuda()
    tab = torch.from_numpy(p.tab).cuda()
    outs = []
    for _ in range(2):
        rho = torch.zeros(p.nset, p.ngrid, dtype=torch.float64, device="cuda")
        cm.aodmao2rho_ex(rho, dms, ao, ao, (p.nao, p.ngrid), (p.nao, p.ngrid), p.nset, tab,
                         p.nblk, p.blksize, precision=cm.PREC_OZAKI_INT8)
        torch.cuda.synchronize()
        outs.append(rho.cpu().numpy())
    assert np.array_equal(outs[0], outs[1])
    assert normwise(outs[0], wl.dense_rho(p.ao, p.ao, p.dms, p.tab, p.blksize)) < TOL


@pytest.mark.parametrize("kind", ["symmetric", "one_entry_off", "general"])
@pytest.mark.parametrize("nao", [296, 600])
def test_split_symmetric_d_mode_and_its_check(cm, oracle, wl, kind, nao):
    """Symmetric D takes the half contraction (row tiles of 128 from their own
    compacted columns on, the diagonal tile's strict upper triangle and half
    diagonal); one differing entry, or a general D, the full one.  The oracle
    never assumes symmetry."""
    p = wl.small_masked(seed=50 + nao, nao=nao, ngrid=2500, blksize=64, nset=2, density=0.5)
    dms = p.dms.copy()
    if kind == "one_entry_off":
        dms[1, 17, nao - 5] += 10.0
    elif kind == "general":
        dms = np.random.default_rng(nao).uniform(-1, 1, dms.shape)
    rho = np.zeros((2, p.ngrid))
    ref = np.zeros((2, p.ngrid))
    args = ((p.nao, p.ngrid), (p.nao, p.ngrid), 2, p.tab, p.nblk, 64)
    split(cm, rho, dms, p.ao, p.ao, *args)
    oracle.aodmao2rho(ref, dms, p.ao, p.ao, *args)
    assert normwise(rho, ref) < TOL
