"""GPU test of cfgmm_aodmao2rho_dev_noalloc, the masked AO-DM-AO entry point
for callers that cannot allocate device memory (a host whose pool owns all of
the GPU's memory, or a loop that must not call cudaMalloc/cudaFree).  It runs
the same kernels as cfgmm_aodmao2rho_dev, with their scratch in a fixed array
inside the library instead of freshly allocated memory.

Called through the C ABI with ctypes; on two calls in a row (different
problems, so the second one starts from the first one's leftover scratch) the
output must match the existing entry point's within the parity tolerance, and
the second call must not change the device's free memory.  The file name makes
pytest collect it last.
"""
import ctypes

import numpy as np
import pytest

from conftest import normwise

pytestmark = pytest.mark.gpu
TOL = 1e-13
NOALLOC_SCRATCH_BYTES = 32 << 20


@pytest.fixture(scope="module")
def capi(cm):
    L = ctypes.CDLL(cm.library_path)
    P, S, I = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int
    L.cfgmm_aodmao2rho_dev_noalloc.argtypes = [P, P, P, P, S, S, S, S, S, P, S, S, P]
    L.cfgmm_aodmao2rho_dev_noalloc.restype = I
    L.cfgmm_aodmao2rho_dev.argtypes = [P, P, P, P, S, S, S, S, S, P, S, S, I, P]
    L.cfgmm_aodmao2rho_dev.restype = I
    L.cfgmm_last_error.restype = ctypes.c_char_p
    return L


def _device_problem(p):
    import torch
    return (torch.from_numpy(p.ao).cuda(), torch.from_numpy(p.dms).cuda(),
            torch.from_numpy(p.tab).cuda())


def _run(capi, fn, p, ao, dms, tab):
    import torch
    rho = torch.zeros(p.nset, p.ngrid, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    args = [rho.data_ptr(), dms.data_ptr(), ao.data_ptr(), ao.data_ptr(), p.nao, p.ngrid, p.nao,
            p.ngrid, p.nset, tab.data_ptr(), p.nblk, p.blksize]
    if fn == "noalloc":
        rc = capi.cfgmm_aodmao2rho_dev_noalloc(*args, stream)
    else:
        rc = capi.cfgmm_aodmao2rho_dev(*args, 0, stream)  # CFGMM_PREC_FP64
    torch.cuda.synchronize()
    assert rc == 0, capi.cfgmm_last_error()
    return rho.cpu().numpy()


def test_noalloc_matches_allocating_entry_point(capi, wl):
    import torch
    problems = [wl.small_masked(seed=7, nao=512, ngrid=4096, nset=3),
                wl.geometric(seed=2, nao=300, nshell=60, natom=15, ngrid=3000, blksize=48,
                             nset=2)]
    for call, p in enumerate(problems):
        ao, dms, tab = _device_problem(p)
        ref = _run(capi, "dev", p, ao, dms, tab)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        got = _run(capi, "noalloc", p, ao, dms, tab)
        free_after = torch.cuda.mem_get_info()[0]
        assert normwise(got, ref) < TOL, f"call {call}"
        assert np.abs(ref).max() > 0
        if call > 0:  # the first call may load the library's device image
            assert free_after == free_before


def test_noalloc_matches_oracle(capi, wl, oracle):
    """An independent check: the no-allocation call against the oracle (the
    CPU restatement of the reference's loops), not only against the other
    entry point."""
    p = wl.small_masked(seed=11, nao=256, ngrid=2048, nset=2)
    ao, dms, tab = _device_problem(p)
    for _ in range(2):  # the second call starts from the first one's leftover scratch
        got = _run(capi, "noalloc", p, ao, dms, tab)
        ref = np.zeros((p.nset, p.ngrid))
        oracle.aodmao2rho(ref, p.dms, p.ao, p.ao, (p.nao, p.ngrid), (p.nao, p.ngrid), p.nset,
                          p.tab, p.nblk, p.blksize)
        assert normwise(got, ref) < TOL


def test_noalloc_refuses_oversized_problem(capi, wl):
    import torch
    nao, ngrid, nset, blk = 4000, 65536, 4, 64  # needs far more than 32 MiB of scratch
    dummy = torch.zeros(1, dtype=torch.float64, device="cuda")
    tab = torch.zeros(1, dtype=torch.uint8, device="cuda")
    rc = capi.cfgmm_aodmao2rho_dev_noalloc(dummy.data_ptr(), dummy.data_ptr(), dummy.data_ptr(),
                                           dummy.data_ptr(), nao, ngrid, nao, ngrid, nset,
                                           tab.data_ptr(), ngrid // blk, blk,
                                           torch.cuda.current_stream().cuda_stream)
    assert rc == -1
    msg = capi.cfgmm_last_error().decode()
    assert "bytes of scratch" in msg and str(NOALLOC_SCRATCH_BYTES) in msg
