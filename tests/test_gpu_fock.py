"""GPU parity tests of the Fock-build contraction (the transpose of AO-DM-AO):
V_s[u,v] += sum_g phi_lhs[u,g] w_s[g] phi_rhs[v,g] over the points whose block
has both u and v active.  Checked against the oracle's restatement of that
formula on the same seeded inputs: ragged and partial blocks, BLKSIZE 16, 48,
64 and 100, a single partial 128-AO tile, padded strides, phi_lhs != phi_rhs,
masked entries holding nonzero phi, accumulation into a nonzero V, nset > 1,
one array passed as both phi_lhs and phi_rhs (the compacted form then forms
half the products and mirrors them),
fully masked tables, device tensors; at a molecule-sized case through the
size-independent identity sum(V(w) * D) == sum(w * rho(D)) with the GPU
AO-DM-AO contraction.  FP64 results within 1e-13 normwise of the oracle."""
import numpy as np
import pytest

from conftest import normwise

pytestmark = pytest.mark.gpu
TOL = 1e-13


def _case(seed, nao, ngrid, nset, blk, pad_ao=0, pad_grid=0, density=0.4, same=False):
    rng = np.random.default_rng(seed)
    sg = ngrid + pad_grid
    nblk = -(-ngrid // blk)
    lhs = rng.standard_normal((nao, sg))  # nonzero under the mask: only the mask excludes them
    rhs = lhs if same else rng.standard_normal((nao, sg))
    ws = rng.uniform(-1, 1, (nset, sg))
    tab = (rng.random((nao, nblk + 1)) < density).astype(np.uint8)  # ldtab = nblk + 1
    vs = rng.uniform(-1, 1, (nset, nao + pad_ao, nao + pad_ao))
    return lhs, rhs, ws, tab, vs, (nao + pad_ao, sg), (nao, ngrid)


@pytest.mark.parametrize("nao,ngrid,nset,blk,pad_ao,pad_grid,same", [
    (100, 1000, 1, 48, 0, 0, True),      # one partial 128-AO tile, last block partial
    (300, 4097, 2, 64, 5, 7, False),     # padded strides, ragged K tail
    (513, 3001, 1, 100, 0, 3, False),    # BLKSIZE not a multiple of the 32-point K step
    (257, 2048, 3, 16, 1, 0, True),      # blocks smaller than a K step
    (40, 10, 1, 16, 0, 0, False),        # fewer points than a K step
    (700, 3000, 2, 64, 2, 1, True),      # one array for both sides: mirrored products
])
def test_fock_matches_oracle(cm, oracle, nao, ngrid, nset, blk, pad_ao, pad_grid, same):
    lhs, rhs, ws, tab, vs, strides, shape = _case(nao + ngrid, nao, ngrid, nset, blk, pad_ao,
                                                  pad_grid, same=same)
    ref = vs.copy()
    oracle.aodm_fock(ref, ws, lhs, rhs, strides, shape, nset, tab, tab.shape[1], blk)
    cm.aodm_fock(vs, ws, lhs, rhs, strides, shape, nset, tab, tab.shape[1], blk)
    assert normwise(vs, ref) < TOL
    if pad_ao:  # padding of V untouched
        assert np.array_equal(vs[:, nao:, :], ref[:, nao:, :])
        assert np.array_equal(vs[:, :, nao:], ref[:, :, nao:])


def test_fock_fully_masked_is_noop(cm):
    lhs, rhs, ws, tab, vs, strides, shape = _case(7, 200, 900, 2, 48)
    tab[:] = 0
    v0 = vs.copy()
    cm.aodm_fock(vs, ws, lhs, rhs, strides, shape, 2, tab, tab.shape[1], 48)
    assert np.array_equal(vs, v0)


def test_fock_sparse_tiles(cm, oracle, wl):
    """Shell-structured mask with whole 128-AO tiles inactive over long grid
    stretches, so that K steps are skipped in some tiles and not in others."""
    p = wl.small_masked(seed=21, nao=768, ngrid=6000, blksize=64, nset=1, density=0.15)
    p.tab[:256, :40] = 0  # the first two tiles idle on the first 2560 points
    rng = np.random.default_rng(21)
    ws = rng.uniform(0, 1, (1, p.ngrid))
    vs = np.zeros((1, p.nao, p.nao))
    ref = vs.copy()
    args = ((p.nao, p.ngrid), (p.nao, p.ngrid), 1, p.tab, p.nblk, p.blksize)
    oracle.aodm_fock(ref, ws, p.ao, p.ao, *args)
    cm.aodm_fock(vs, ws, p.ao, p.ao, *args)
    assert normwise(vs, ref) < TOL


def test_fock_device_tensors(cm, oracle):
    import torch
    lhs, rhs, ws, tab, vs, strides, shape = _case(11, 333, 2500, 2, 48, pad_ao=2, pad_grid=4)
    ref = vs.copy()
    oracle.aodm_fock(ref, ws, lhs, rhs, strides, shape, 2, tab, tab.shape[1], 48)
    d = {k: torch.from_numpy(x).cuda() for k, x in
         dict(lhs=lhs, rhs=rhs, ws=ws, tab=tab, vs=vs).items()}
    cm.aodm_fock(d["vs"], d["ws"], d["lhs"], d["rhs"], strides, shape, 2, d["tab"],
                 tab.shape[1], 48)
    torch.cuda.synchronize()
    assert normwise(d["vs"].cpu().numpy(), ref) < TOL


def test_fock_is_the_adjoint_of_aodmao2rho(cm, wl):
    """sum_uv V(w)[u,v] D[u,v] == sum_g w[g] rho(D)[g], both from the GPU, on a
    molecule-sized case (2048 AOs, 16384 points in blocks of 64)."""
    p = wl.small_masked(seed=31, nao=2048, shell=8, ngrid=16384, blksize=64, nset=1)
    w = np.random.default_rng(31).uniform(-1, 1, (1, p.ngrid))
    rho = np.zeros((1, p.ngrid))
    args = ((p.nao, p.ngrid), (p.nao, p.ngrid), 1, p.tab, p.nblk)
    cm.aodmao2rho_ex(rho, p.dms, p.ao, p.ao, *args, blksize=p.blksize)
    v = np.zeros((1, p.nao, p.nao))
    cm.aodm_fock(v, w, p.ao, p.ao, *args, blksize=p.blksize)
    scale = float(np.sum(np.abs(v) * np.abs(p.dms)))
    assert abs(float(np.sum(v * p.dms)) - float(np.sum(w * rho))) <= 1e-13 * scale
    assert np.allclose(v[0], v[0].T, rtol=0, atol=1e-12 * np.abs(v).max())  # phi_lhs == phi_rhs


def test_fock_compacted_and_dense_forms_agree(cm, oracle):
    """The compacted form (per-block active lists, V scattered by FP64 atomics)
    and the dense product with K-step skipping (CFGMM_FOCK_DENSE=1) on the same
    inputs, both within 1e-13 of the oracle."""
    import os, subprocess, sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    tmp = os.environ.get("TMPDIR", "/tmp")
    code = ("import importlib,sys,numpy as np; sys.path.insert(0,'.'); sys.path.insert(0,'tests');"
            "cm=importlib.import_module('cfgable-matmul_b200');"
            "from test_gpu_fock import _case;"
            "lhs,rhs,ws,tab,vs,st,sh=_case(77,700,3000,2,64,pad_ao=2,pad_grid=1);"
            "cm.aodm_fock(vs,ws,lhs,rhs,st,sh,2,tab,tab.shape[1],64); np.save(sys.argv[1], vs)")
    outs = []
    for dense in ("0", "1"):
        path = os.path.join(tmp, f"cfgmm_fock_dense{dense}.npy")
        subprocess.run([sys.executable, "-c", code, path], cwd=root, check=True,
                       env=dict(os.environ, CFGMM_FOCK_DENSE=dense))
        outs.append(np.load(path))
    lhs, rhs, ws, tab, vs, strides, shape = _case(77, 700, 3000, 2, 64, pad_ao=2, pad_grid=1)
    oracle.aodm_fock(vs, ws, lhs, rhs, strides, shape, 2, tab, tab.shape[1], 64)
    for o in outs:
        assert normwise(o, vs) < TOL
