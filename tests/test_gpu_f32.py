"""GPU tests of the f32 forms of the two paths (MatmulLoops<f32>: the reference
is generic over T but implements f64 only, src/structs.rs:19-20).  f32 inputs,
f64 arithmetic on the device (DMMA or the Ozaki split with the moduli that
26-bit operands need), one rounding to f32: results within 1e-7 normwise (FP64)
and 2e-7 (split) of the f64 result on the same f32 inputs, i.e. at the f32
rounding of the output."""
import numpy as np
import pytest

from conftest import normwise

pytestmark = pytest.mark.gpu


def _op(x, t):
    return x.T if t else x


@pytest.mark.parametrize("prec,tol", [(0, 1e-7), (1, 2e-7)])
@pytest.mark.parametrize("transa,transb", [(False, False), (False, True), (True, False),
                                           (True, True)])
@pytest.mark.parametrize("m,n,k,pad", [(300, 500, 400, 0), (1037, 1161, 1999, 3)])
def test_matmul_f32(cm, prec, tol, transa, transb, m, n, k, pad):
    rng = np.random.default_rng(m + k + 2 * transa + transb)
    ar, ac = (k, m) if transa else (m, k)
    br, bc = (n, k) if transb else (k, n)
    a = rng.uniform(-1, 1, (ar, ac + pad)).astype(np.float32)
    b = rng.uniform(-1, 1, (br, bc + 2 * pad)).astype(np.float32)
    c = rng.uniform(-1, 1, (m, n + pad)).astype(np.float32)
    ref = c.astype(np.float64)
    ref[:, :n] += _op(a[:, :ac].astype(np.float64), transa) @ _op(b[:, :bc].astype(np.float64),
                                                                 transb)
    c0 = c.copy()
    cm.matmul_f32(c, a, b, m, n, k, ac + pad, bc + 2 * pad, n + pad, transa, transb,
                  precision=prec)
    assert normwise(c[:, :n].astype(np.float64), ref[:, :n]) < tol
    assert np.array_equal(c[:, n:], c0[:, n:])  # padding untouched


@pytest.mark.parametrize("prec,tol", [(0, 1e-7), (1, 2e-7)])
def test_aodmao2rho_f32(cm, oracle, wl, prec, tol):
    p = wl.small_masked(seed=61, nao=512, ngrid=4000, blksize=64, nset=2)
    lhs = p.ao.astype(np.float32)
    dms = p.dms.astype(np.float32)
    rho = np.random.default_rng(61).uniform(-1, 1, (2, p.ngrid)).astype(np.float32)
    ref = rho.astype(np.float64)
    args = ((p.nao, p.ngrid), (p.nao, p.ngrid), 2, p.tab, p.nblk)
    oracle.aodmao2rho(ref, dms.astype(np.float64), lhs.astype(np.float64), lhs.astype(np.float64),
                      *args, 64)
    cm.aodmao2rho_f32(rho, dms, lhs, lhs, *args, blksize=64, precision=prec)
    assert normwise(rho.astype(np.float64), ref) < tol


def test_f32_device_tensors(cm, oracle, wl):
    import torch
    p = wl.small_masked(seed=62, nao=256, ngrid=2048, blksize=64, nset=1)
    lhs = p.ao.astype(np.float32)
    rhs = (p.ao * 0.5).astype(np.float32)  # phi_lhs != phi_rhs
    dms = p.dms.astype(np.float32)
    ref = np.zeros((1, p.ngrid))
    args = ((p.nao, p.ngrid), (p.nao, p.ngrid), 1, p.tab, p.nblk)
    oracle.aodmao2rho(ref, dms.astype(np.float64), lhs.astype(np.float64), rhs.astype(np.float64),
                      *args, 64)
    t = {k: torch.from_numpy(v).cuda() for k, v in dict(lhs=lhs, rhs=rhs, dms=dms, tab=p.tab).items()}
    rho = torch.zeros(1, p.ngrid, dtype=torch.float32, device="cuda")
    cm.aodmao2rho_f32(rho, t["dms"], t["lhs"], t["rhs"], *args[:2], 1, t["tab"], p.nblk, 64)
    a = torch.rand(200, 300, dtype=torch.float32, device="cuda")
    b = torch.rand(300, 100, dtype=torch.float32, device="cuda")
    c = torch.zeros(200, 100, dtype=torch.float32, device="cuda")
    cm.matmul_f32(c, a, b, 200, 100, 300, 300, 100, 100, False, False)
    torch.cuda.synchronize()
    assert normwise(rho.cpu().numpy().astype(np.float64), ref) < 1e-7
    cref = a.double().cpu().numpy() @ b.double().cpu().numpy()
    assert normwise(c.cpu().numpy().astype(np.float64), cref) < 1e-7
