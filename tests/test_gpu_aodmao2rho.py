"""GPU parity tests of the masked AO-DM-AO contraction through the C ABI.

Named after and built from the reference's tests (test_aodmao2rho_1 and
test_aodmao2rho_all_dense, src/impl_aodmao2rho.rs:263-425: two different phi
tables, a non-symmetric D, an odd ngrid with a partial block); plus the edge
cases the reference's loops handle: empty blocks, fully masked tables, ragged
blocks, padded strides, nset > 1, masked entries holding nonzero phi.  FP64
results must be within 1e-13 normwise of the oracle.
"""
import numpy as np
import pytest

from conftest import load_golden, normwise

pytestmark = pytest.mark.gpu
TOL = 1e-13


def run_gpu(cm, rho, dms, lhs, rhs, strides, shape, nset, tab, ldtab, blk):
    cm.MatmulLoops().aodmao2rho_loop_parallel(rho, dms, lhs, rhs, strides, shape, nset, tab, ldtab,
                                              BLKSIZE=blk)


def run_oracle(oracle, rho, dms, lhs, rhs, strides, shape, nset, tab, ldtab, blk):
    oracle.aodmao2rho(rho, dms, lhs, rhs, strides, shape, nset, tab, ldtab, blk)


@pytest.mark.parametrize("name", ["aodmao2rho_pattern25", "aodmao2rho_all_dense",
                                  "aodmao2rho_pattern25_nset2_blk64"])
def test_aodmao2rho_golden(cm, wl, name):
    g = load_golden(name)
    nao, ngrid, nset, blk = int(g["nao"]), int(g["ngrid"]), int(g["nset"]), int(g["blksize"])
    lhs, rhs, dm, tab, nblk = wl.ref_aodmao2rho_inputs(nao, ngrid, nset, blk, bool(g["dense"]))
    rho = np.zeros((nset, ngrid))
    if blk == 48:
        cm.aodmao2rho_anyway(rho, dm, lhs, rhs, (nao, ngrid), (nao, ngrid), nset, tab, nblk)
    else:
        run_gpu(cm, rho, dm, lhs, rhs, (nao, ngrid), (nao, ngrid), nset, tab, nblk, blk)
    assert normwise(rho, g["rho"]) < TOL


@pytest.mark.parametrize("dense", [False, True])
def test_aodmao2rho_1_reference_shape(cm, oracle, wl, dense):
    """test_aodmao2rho_1 / _all_dense at a reduced nao (ngrid 131073 as in the
    reference: 2731 blocks of 48, the last one partial)."""
    nao, ngrid = 260, 131073
    lhs, rhs, dm, tab, nblk = wl.ref_aodmao2rho_inputs(nao, ngrid, 1, 48, dense)
    rho = np.zeros((1, ngrid))
    ref = np.zeros((1, ngrid))
    cm.aodmao2rho_anyway(rho, dm, lhs, rhs, (nao, ngrid), (nao, ngrid), 1, tab, nblk)
    run_oracle(oracle, ref, dm, lhs, rhs, (nao, ngrid), (nao, ngrid), 1, tab, nblk, 48)
    assert normwise(rho, ref) < TOL


def test_small_bernoulli_workload(cm, oracle, wl):
    """512 AOs in 64 shells of 8, 4096 points in blocks of 64, 1 DM, density 0.3."""
    p = wl.small_masked(seed=0)
    rho = np.zeros((1, p.ngrid))
    ref = np.zeros((1, p.ngrid))
    args = ((p.nao, p.ngrid), (p.nao, p.ngrid), 1, p.tab, p.nblk, p.blksize)
    run_gpu(cm, rho, p.dms, p.ao, p.ao, *args)
    run_oracle(oracle, ref, p.dms, p.ao, p.ao, *args)
    assert normwise(rho, ref) < TOL


def test_geometric_taxol_size(cm, oracle, wl):
    """2228 AOs, 16384 points in blocks of 64, 3 DMs, tile density 0.3."""
    p = wl.geometric(seed=0)
    rho = np.zeros((p.nset, p.ngrid))
    ref = np.zeros((p.nset, p.ngrid))
    args = ((p.nao, p.ngrid), (p.nao, p.ngrid), p.nset, p.tab, p.nblk, p.blksize)
    run_gpu(cm, rho, p.dms, p.ao, p.ao, *args)
    run_oracle(oracle, ref, p.dms, p.ao, p.ao, *args)
    assert normwise(rho, ref) < TOL


@pytest.mark.parametrize("blk", [1, 16, 48, 64, 100, 128, 200])
@pytest.mark.parametrize("nset", [1, 2, 3, 4, 5])
def test_ragged_blocks_and_sets(cm, oracle, wl, blk, nset):
    rng = np.random.default_rng(blk * 10 + nset)
    nao, ngrid = 157, 1001
    nblk = -(-ngrid // blk)
    lhs = rng.standard_normal((nao, ngrid))
    rhs = rng.standard_normal((nao, ngrid))  # masked entries stay nonzero on purpose
    dms = rng.uniform(-1, 1, (nset, nao, nao))  # non-symmetric
    tab = (rng.random((nao, nblk)) < 0.35).astype(np.uint8)
    tab[:, nblk // 2] = 0  # an empty block
    rho0 = rng.standard_normal((nset, ngrid))
    rho, ref = rho0.copy(), rho0.copy()
    gpu_args = ((nao, ngrid), (nao, ngrid), nset, tab, nblk, blk)
    if blk % 16 == 0:
        run_gpu(cm, rho, dms, lhs, rhs, *gpu_args)
        run_oracle(oracle, ref, dms, lhs, rhs, *gpu_args)
        assert normwise(rho, ref) < TOL
    else:  # the oracle (like the reference) needs BLKSIZE % 16 == 0: use dense numpy
        run_gpu(cm, rho, dms, lhs, rhs, *gpu_args)
        ref = rho0 + wl.dense_rho(lhs, rhs, dms, tab, blk)
        assert normwise(rho, ref) < TOL
    # the empty block is untouched bit for bit
    g0, g1 = (nblk // 2) * blk, min((nblk // 2 + 1) * blk, ngrid)
    assert np.array_equal(rho[:, g0:g1], rho0[:, g0:g1])


def test_fully_masked_table_leaves_rho_untouched(cm):
    nao, ngrid, blk = 64, 300, 48
    nblk = -(-ngrid // blk)
    rho = np.full((2, ngrid), -0.0)
    ones = np.ones((nao, ngrid))
    cm.aodmao2rho_anyway(rho, np.ones((2, nao, nao)), ones, ones, (nao, ngrid), (nao, ngrid), 2,
                         np.zeros((nao, nblk), np.uint8), nblk)
    assert np.all(np.signbit(rho))  # not even -0.0 -> +0.0


def test_padded_strides(cm, oracle):
    rng = np.random.default_rng(9)
    nao, ngrid, nset, blk = 120, 700, 2, 64
    sa, sg = nao + 9, ngrid + 11
    nblk = -(-ngrid // blk)
    ldtab = nblk + 3
    lhs = rng.standard_normal((nao, sg))
    dms = rng.uniform(-1, 1, (nset, sa, sa))
    tab = (rng.random((nao, ldtab)) < 0.4).astype(np.uint8)
    rho = np.zeros((nset, sg))
    ref = np.zeros((nset, sg))
    args = ((sa, sg), (nao, ngrid), nset, tab, ldtab, blk)
    run_gpu(cm, rho, dms, lhs, lhs, *args)
    run_oracle(oracle, ref, dms, lhs, lhs, *args)
    assert normwise(rho, ref) < TOL
    assert np.all(rho[:, ngrid:] == 0.0)


def test_device_pointers_and_determinism(cm, wl):
    import torch
    p = wl.small_masked(seed=4, nset=3)
    ao = torch.from_numpy(p.ao).cuda()
    dms = torch.from_numpy(p.dms).cuda()
    tab = torch.from_numpy(p.tab).cuda()
    outs = []
    for _ in range(2):
        rho = torch.zeros(p.nset, p.ngrid, dtype=torch.float64, device="cuda")
        cm.aodmao2rho_ex(rho, dms, ao, ao, (p.nao, p.ngrid), (p.nao, p.ngrid), p.nset, tab,
                         p.nblk, p.blksize)
        torch.cuda.synchronize()
        outs.append(rho.cpu().numpy())
    assert np.array_equal(outs[0], outs[1])  # fixed reduction order
    ref = wl.dense_rho(p.ao, p.ao, p.dms, p.tab, p.blksize)
    assert normwise(outs[0], ref) < TOL


@pytest.mark.parametrize("stride_pad", [0, 1])
def test_pipelined_and_plain_forms_agree(cm, oracle, stride_pad):
    """The pipelined kernel and the form it replaces, forced with
    CFGMM_AODM_PIPE=0, on the same inputs; the pipelined kernel fetches the
    phi rows by TMA gather4 when they are 16-byte aligned (stride_pad 0) and
    by cp.async otherwise (stride_pad 1).  Both within 1e-13 of the oracle."""
    import json, os, subprocess, sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    tmp = os.environ.get("TMPDIR", "/tmp")
    code = ("import importlib,sys,numpy as np; sys.path.insert(0,'.');"
            "cm=importlib.import_module('cfgable-matmul_b200');"
            "wl=importlib.import_module('cfgable-matmul_b200.workloads');"
            "pad=int(sys.argv[2]); p=wl.small_masked(seed=9,nao=768,ngrid=5000,blksize=64,nset=3);"
            "sg=p.ngrid+pad; ao=np.zeros((p.nao,sg)); ao[:,:p.ngrid]=p.ao;"
            "rho=np.zeros((p.nset,sg)); "
            "cm.aodmao2rho_ex(rho,p.dms,ao,ao,(p.nao,sg),(p.nao,p.ngrid),p.nset,p.tab,p.nblk,64);"
            "np.save(sys.argv[1], rho)")
    outs = []
    for pipe in ("1", "0"):
        path = os.path.join(tmp, f"cfgmm_aodm_pipe{pipe}_{stride_pad}.npy")
        env = dict(os.environ, CFGMM_AODM_PIPE=pipe)
        subprocess.run([sys.executable, "-c", code, path, str(stride_pad)], cwd=root, env=env,
                       check=True)
        outs.append(np.load(path))
    wl = __import__("importlib").import_module("cfgable-matmul_b200.workloads")
    p = wl.small_masked(seed=9, nao=768, ngrid=5000, blksize=64, nset=3)
    ref = np.zeros((p.nset, p.ngrid))
    oracle.aodmao2rho(ref, p.dms, p.ao, p.ao, (p.nao, p.ngrid), (p.nao, p.ngrid), p.nset, p.tab,
                      p.nblk, 64)
    for o in outs:
        assert normwise(o[:, :p.ngrid], ref) < TOL
    assert normwise(outs[0], outs[1]) < 1e-14


@pytest.mark.parametrize("kind", ["symmetric", "one_entry_off", "general"])
@pytest.mark.parametrize("nset", [1, 3])
def test_symmetric_d_mode_and_its_check(cm, oracle, kind, nset):
    """The pipelined form contracts only the upper half of D when every D_s
    equals its transpose bit for bit (checked on the device each call); one
    differing entry, or a general D, must take the full contraction.  The
    oracle never assumes symmetry, so a wrongly taken symmetric mode fails."""
    rng = np.random.default_rng(40 + nset)
    from importlib import import_module
    wl = import_module("cfgable-matmul_b200.workloads")
    p = wl.small_masked(seed=40 + nset, nao=600, ngrid=3000, blksize=64, nset=nset, density=0.5)
    dms = p.dms.copy()
    if kind == "one_entry_off":
        dms[nset - 1, 17, 411] += 10.0  # D[17][411] != D[411][17]; both active in ~1/4 of blocks
    elif kind == "general":
        dms = rng.uniform(-1, 1, dms.shape)
    tab = p.tab
    rho = np.zeros((nset, p.ngrid))
    ref = np.zeros((nset, p.ngrid))
    args = ((p.nao, p.ngrid), (p.nao, p.ngrid), nset, tab, p.nblk)
    cm.aodmao2rho_ex(rho, dms, p.ao, p.ao, *args, blksize=64)
    oracle.aodmao2rho(ref, dms, p.ao, p.ao, *args, 64)
    assert normwise(rho, ref) < TOL


@pytest.mark.parametrize("prec", [0, 1])
def test_large_host_call_in_blocks(cm, oracle, prec):
    """A host-pointer call whose phi table exceeds 64 MB runs in blocks of grid
    blocks whose transfers overlap the work: the same bits as one
    device-pointer call (each grid block is contracted alike), accumulation
    into a nonzero rho, padded strides, phi_lhs != phi_rhs, and the oracle's
    result within the parity tolerance."""
    import torch
    nao, ngrid, nset, blk = 1100, 8000, 2, 64
    sa, sg = nao + 3, ngrid + 5
    rng = np.random.default_rng(77 + prec)
    nblk = -(-ngrid // blk)
    tab = (rng.random((nao, nblk + 1)) < 0.35).astype(np.uint8)
    lhs = rng.standard_normal((nao, sg))
    rhs = rng.standard_normal((nao, sg))
    a = rng.uniform(-1, 1, (nset, sa, sa))
    dms = np.ascontiguousarray(0.5 * (a + a.transpose(0, 2, 1)))
    rho0 = rng.uniform(-1, 1, (nset, sg))
    rho = rho0.copy()
    cm.aodmao2rho_ex(rho, dms, lhs, rhs, (sa, sg), (nao, ngrid), nset, tab, tab.shape[1], blk, prec)
    d = {k: torch.from_numpy(np.ascontiguousarray(x)).cuda()
         for k, x in dict(rho=rho0, dms=dms, lhs=lhs, rhs=rhs, tab=tab).items()}
    cm.aodmao2rho_ex(d["rho"], d["dms"], d["lhs"], d["rhs"], (sa, sg), (nao, ngrid), nset, d["tab"],
                     tab.shape[1], blk, prec)
    torch.cuda.synchronize()
    assert np.array_equal(d["rho"].cpu().numpy(), rho)
    ref = rho0.copy()
    oracle.aodmao2rho(ref, dms, lhs, rhs, (sa, sg), (nao, ngrid), nset, tab, tab.shape[1], blk)
    assert normwise(rho, ref) < (1e-12 if prec else 1e-13)
    assert np.array_equal(rho[:, ngrid:], rho0[:, ngrid:])  # padding of rho untouched


@pytest.mark.parametrize("prec", [0, 1])
def test_symmetric_d_with_two_phi_arrays(cm, oracle, prec):
    """A symmetric D with phi_lhs != phi_rhs: the half contraction of the
    symmetric mode does not apply (it needs one phi array for both sides), so
    the full contraction runs; checked against the oracle."""
    nao, ngrid, nset, blk = 300, 2000, 2, 64
    rng = np.random.default_rng(91 + prec)
    nblk = -(-ngrid // blk)
    tab = (rng.random((nao, nblk)) < 0.4).astype(np.uint8)
    lhs = rng.standard_normal((nao, ngrid))
    rhs = rng.standard_normal((nao, ngrid))
    a = rng.uniform(-1, 1, (nset, nao, nao))
    dms = np.ascontiguousarray(0.5 * (a + a.transpose(0, 2, 1)))
    rho = np.zeros((nset, ngrid))
    ref = rho.copy()
    cm.aodmao2rho_ex(rho, dms, lhs, rhs, (nao, ngrid), (nao, ngrid), nset, tab, nblk, blk, prec)
    oracle.aodmao2rho(ref, dms, lhs, rhs, (nao, ngrid), (nao, ngrid), nset, tab, nblk, blk)
    assert normwise(rho, ref) < (1e-12 if prec else 1e-13)
