"""GPU tests of the AO evaluator and the mask builder (cfgmm_eval_ao_dev,
cfgmm_mask_ao_dev) against numpy, and of the device-built workload through
the contraction against the oracle."""
import numpy as np
import pytest

from conftest import normwise

pytestmark = pytest.mark.gpu


def _small(wl, seed=0):
    mol = wl.molecule(seed, nao=120, nshell=24, natom=8, box_angstrom=6.0)
    pts = wl.grid_points(np.random.default_rng(seed), mol, 1000, 64)
    return mol, pts


def test_eval_ao_matches_numpy(cm, wl):
    import torch
    mol, pts = _small(wl)
    d = wl.DeviceMolecule(mol)
    ngrid = len(pts)
    ao = torch.full((mol.nao, ngrid + 5), 7.0, dtype=torch.float64, device="cuda")  # padded
    bmax = torch.empty(mol.nshell, -(-ngrid // 64), dtype=torch.float64, device="cuda")
    p = torch.from_numpy(pts).cuda()
    cm.lib()
    rc = cm.lib().cfgmm_eval_ao_dev(ao.data_ptr(), ngrid + 5, p.data_ptr(), ngrid,
                                    d.xyz.data_ptr(), d.l.data_ptr(), d.alpha.data_ptr(),
                                    d.norm.data_ptr(), d.row.data_ptr(), mol.nshell,
                                    bmax.data_ptr(), 64, torch.cuda.current_stream().cuda_stream)
    assert rc == 0
    ref = wl.eval_ao_numpy(mol, pts)
    got = ao.cpu().numpy()
    assert np.abs(got[:, :ngrid] - ref).max() <= 1e-13 * np.abs(ref).max()
    assert (got[:, ngrid:] == 7.0).all()  # padding untouched
    # exp(-x) for x up to ~700 carries a relative error of about x ulp
    assert np.allclose(bmax.cpu().numpy(), wl.shell_block_max(mol, ref, 64), rtol=1e-11, atol=0)


def test_mask_matches_numpy_and_contracts(cm, wl, oracle):
    import torch
    mol, pts = _small(wl, 3)
    d = wl.DeviceMolecule(mol)
    ao, tab = wl.device_grid(cm, d, pts, 64, 0.4)
    ref = wl.eval_ao_numpy(mol, pts)
    shmax = wl.shell_block_max(mol, ref, 64)
    thr = float(torch.quantile(torch.from_numpy(shmax).flatten(), 0.6))
    ref_tab = np.repeat((shmax > thr).astype(np.uint8), mol.sizes, axis=0)
    got_tab = tab.cpu().numpy()
    # a max within rounding of the threshold may fall either side
    near = np.repeat(np.abs(shmax - thr) <= 1e-12 * thr, mol.sizes, axis=0)
    assert ((got_tab == ref_tab) | near).all()
    ref[~wl.expand_mask(got_tab, len(pts), 64)] = 0.0
    got = ao.cpu().numpy()
    assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max()
    # the contraction on the device-built inputs
    dms = wl.sym_dms(np.random.default_rng(5), 2, mol.nao)
    nblk = got_tab.shape[1]
    rho = torch.zeros(2, len(pts), dtype=torch.float64, device="cuda")
    cm.aodmao2rho_ex(rho, torch.from_numpy(dms).cuda(), ao, ao, (mol.nao, len(pts)),
                     (mol.nao, len(pts)), 2, tab, nblk, 64)
    out = np.zeros((2, len(pts)))
    oracle.aodmao2rho(out, dms, got, got, (mol.nao, len(pts)), (mol.nao, len(pts)), 2, got_tab,
                      nblk, 64)
    assert normwise(rho.cpu().numpy(), out) < 1e-13


def test_batched_uneven_generator(cm, wl):
    p = wl.batched_uneven(cm, seed=0, nbatch=4, nao=120, nshell=24, natom=8, gmin=64, gmax=512)
    assert len(p.batches) == 4
    for ao, tab, ngrid, nset, dens in p.batches:
        assert ao.shape == (120, ngrid) and 1 <= nset <= 3
        assert 0.0 <= tab.float().mean().item() <= 1.0
