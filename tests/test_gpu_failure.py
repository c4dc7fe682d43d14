"""GPU tests of the failure detection of the tensor-core pipelines, with the
failure made on the host side of the kernel's protocol and never by a fault:
cfgmm_test_arm_wait_timeout arms the next contraction so that one producer
never publishes the first pipeline stage (a flag that nothing sets) and every
wait gives up after a few milliseconds.  The waiting warp records a timeout,
the kernel drains its copies, frees its tensor memory and returns; the call
reports CFGMM_ERR_TIMEOUT, and the next call on the same context runs
normally and matches the oracle.  Covered: the pipelined FP64 kernel
(DMMA, mbarrier ring) and the split pair kernel (tcgen05 + TMEM)."""
import ctypes

import numpy as np
import pytest

from conftest import normwise

pytestmark = pytest.mark.gpu
TOL = {0: 1e-13, 1: 1e-12}
TIMEOUT = -6


@pytest.fixture(scope="module")
def capi(cm):
    L = ctypes.CDLL(cm.library_path)
    P, S, I = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int
    L.cfgmm_aodmao2rho_dev.argtypes = [P, P, P, P, S, S, S, S, S, P, S, S, I, P]
    L.cfgmm_aodmao2rho_dev.restype = I
    L.cfgmm_test_arm_wait_timeout.argtypes = [I, ctypes.c_double]
    L.cfgmm_test_arm_wait_timeout.restype = I
    L.cfgmm_device_check.restype = I
    L.cfgmm_last_error.restype = ctypes.c_char_p
    return L


@pytest.fixture(autouse=True)
def pair_form(monkeypatch):
    # the split hook is taken by the pair kernel
    monkeypatch.setenv("CFGMM_SPLIT_FORM", "pair")


def _problem(wl):
    return wl.small_masked(seed=3, nao=256, ngrid=2048, nset=2)


def _ref(oracle, p):
    ref = np.zeros((p.nset, p.ngrid))
    oracle.aodmao2rho(ref, p.dms, p.ao, p.ao, (p.nao, p.ngrid), (p.nao, p.ngrid), p.nset, p.tab,
                      p.nblk, p.blksize)
    return ref


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64_pipe", "split_pair"])
def test_device_call_times_out_then_recovers(capi, wl, oracle, precision):
    import torch
    p = _problem(wl)
    ao = torch.from_numpy(p.ao).cuda()
    dms = torch.from_numpy(p.dms).cuda()
    tab = torch.from_numpy(p.tab).cuda()
    rho = torch.zeros(p.nset, p.ngrid, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream

    def call():
        return capi.cfgmm_aodmao2rho_dev(rho.data_ptr(), dms.data_ptr(), ao.data_ptr(),
                                         ao.data_ptr(), p.nao, p.ngrid, p.nao, p.ngrid, p.nset,
                                         tab.data_ptr(), p.nblk, p.blksize, precision, stream)

    assert capi.cfgmm_device_check() == 0
    assert capi.cfgmm_test_arm_wait_timeout(precision, 20.0) == 0
    assert call() == 0  # enqueued: a _dev call does not synchronise
    rc = capi.cfgmm_device_check()
    assert rc == TIMEOUT, capi.cfgmm_last_error()
    assert b"timed out" in capi.cfgmm_last_error()
    assert capi.cfgmm_device_check() == 0  # reported once, then cleared
    # the context is intact: the next calls run normally
    for _ in range(2):
        rho.zero_()
        assert call() == 0
        assert capi.cfgmm_device_check() == 0, capi.cfgmm_last_error()
        assert normwise(rho.cpu().numpy(), _ref(oracle, p)) < TOL[precision]


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64_pipe", "split_pair"])
def test_host_call_reports_timeout_then_recovers(cm, capi, wl, oracle, precision):
    p = _problem(wl)
    args = ((p.nao, p.ngrid), (p.nao, p.ngrid), p.nset, p.tab, p.nblk, p.blksize, precision)
    rho = np.zeros((p.nset, p.ngrid))
    assert capi.cfgmm_test_arm_wait_timeout(precision, 15.0) == 0
    with pytest.raises(cm.CfgmmError) as e:
        cm.aodmao2rho_ex(rho, p.dms, p.ao, p.ao, *args)
    assert e.value.status == TIMEOUT
    rho = np.zeros((p.nset, p.ngrid))
    cm.aodmao2rho_ex(rho, p.dms, p.ao, p.ao, *args)
    assert normwise(rho, _ref(oracle, p)) < TOL[precision]
