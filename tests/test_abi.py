"""CPU tests of the C-ABI boundary (libcfgmm.so): it loads, it exports every
symbol include/*.h declares, and it rejects -- before touching any device --
every call the reference would panic on.  No compute call is made here."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

from conftest import ROOT, has_cuda


def _declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(cfgmm_\w+)\s*\(", text))
    return sorted(names)


def test_library_builds_and_loads(cm):
    lib = cm.lib()
    assert os.path.exists(cm.library_path)
    assert lib.cfgmm_version() >= 100


def test_every_declared_symbol_is_exported(cm):
    names = _declared_symbols()
    assert len(names) >= 13
    lib = ctypes.CDLL(cm.library_path)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_status_strings(cm):
    lib = cm.lib()
    for rc in range(0, -8, -1):
        assert lib.cfgmm_status_string(rc)
    assert b"unknown" in lib.cfgmm_status_string(-99)


def _gemm_args(m=4, n=5, k=6):
    a = np.ones((m, k))
    b = np.ones((k, n))
    c = np.zeros((m, n))
    return c, a, b


def test_gemm_short_slice_is_rejected(cm):
    c, a, b = _gemm_args()
    with pytest.raises(ValueError, match="slice too short"):
        cm.matmul_anyway_full(c, a[:3], b, 4, 5, 6, 6, 5, 5, False, False)
    with pytest.raises(ValueError, match="slice too short"):
        cm.matmul_anyway_full(c, a, b, 4, 5, 6, 7, 5, 5, False, False)  # lda 7 overruns A
    with pytest.raises(ValueError, match="slice too short"):
        cm.matmul_anyway_full(c[:2], a, b, 4, 5, 6, 6, 5, 5, False, False)
    with pytest.raises(ValueError):
        cm.matmul_anyway_full(c, a, b, 4, 5, 6, 6, 5, 4, False, False)  # ldc < n
    assert np.all(c == 0)


def test_gemm_zero_sizes_are_noops(cm):
    # The reference's task loops are empty for m, n or k == 0: nothing is
    # touched and no device is needed.
    c, a, b = _gemm_args()
    for m, n, k in ((0, 5, 6), (4, 0, 6), (4, 5, 0)):
        cm.matmul_anyway_full(c, a, b, m, n, k, 6, 5, 5, False, False)
    assert np.all(c == 0)


def test_masked_gemm_transb_panics_first(cm):
    # impl_matmul_non0tab.rs:228-230: transb panics before anything else, even
    # for a zero-sized problem; no device is touched.
    c = np.zeros((2, 2))
    with pytest.raises(NotImplementedError):
        cm.matmul_anyway_full_non0tab(c, np.ones((2, 2)), np.ones((2, 2)), 0, 0, 0, 2, 2, 2,
                                      False, True, np.ones((2, 1), np.uint8), 1)


def test_masked_gemm_short_tab(cm):
    c, a, b = _gemm_args()
    with pytest.raises(ValueError, match="slice too short"):
        cm.matmul_anyway_full_non0tab(c, a, b, 4, 5, 6, 6, 5, 5, False, False,
                                      np.ones(3, np.uint8), 1)


def test_unknown_precision(cm):
    c, a, b = _gemm_args()
    with pytest.raises(ValueError, match="precision"):
        cm.matmul_ex(c, a, b, 4, 5, 6, 6, 5, 5, False, False, precision=7)


def _aodm_args(nao=10, ngrid=100, nset=2, blk=48):
    nblk = -(-ngrid // blk)
    rho = np.zeros((nset, ngrid))
    dms = np.ones((nset, nao, nao))
    ao = np.ones((nao, ngrid))
    tab = np.ones((nao, nblk), np.uint8)
    return rho, dms, ao, tab, nblk


def test_aodm_validation(cm):
    rho, dms, ao, tab, nblk = _aodm_args()
    with pytest.raises(ValueError, match="slice too short"):
        cm.aodmao2rho_anyway(rho, dms[:1], ao, ao, (10, 100), (10, 100), 2, tab, nblk)
    with pytest.raises(ValueError, match="slice too short"):
        cm.aodmao2rho_anyway(rho, dms, ao, ao, (10, 100), (10, 100), 2, tab[:5], nblk)
    with pytest.raises(ValueError, match="slice too short"):
        cm.aodmao2rho_anyway(rho[:1], dms, ao, ao, (10, 100), (10, 100), 2, tab, nblk)
    with pytest.raises(ValueError, match="BLKSIZE"):
        cm.aodmao2rho_ex(rho, dms, ao, ao, (10, 100), (10, 100), 2, tab, nblk, blksize=0)
    with pytest.raises(ValueError, match="stride_grid"):
        cm.aodmao2rho_anyway(rho, dms, ao, ao, (10, 50), (10, 100), 2, tab, nblk)
    assert np.all(rho == 0)


def test_aodm_zero_sizes_are_noops(cm):
    rho, dms, ao, tab, nblk = _aodm_args()
    cm.aodmao2rho_anyway(rho, dms, ao, ao, (10, 100), (0, 100), 2, tab, nblk)
    cm.aodmao2rho_anyway(rho, dms, ao, ao, (10, 100), (10, 0), 2, tab, nblk)
    cm.aodmao2rho_anyway(rho, dms, ao, ao, (10, 100), (10, 100), 0, tab, nblk)
    assert np.all(rho == 0)


def test_fock_validation(cm):
    """The Fock-build call takes V in D's place and w in rho's: the same checks."""
    w, v, ao, tab, nblk = _aodm_args()
    with pytest.raises(ValueError, match="slice too short"):
        cm.aodm_fock(v[:1], w, ao, ao, (10, 100), (10, 100), 2, tab, nblk)
    with pytest.raises(ValueError, match="slice too short"):
        cm.aodm_fock(v, w[:1], ao, ao, (10, 100), (10, 100), 2, tab, nblk)
    with pytest.raises(ValueError, match="slice too short"):
        cm.aodm_fock(v, w, ao, ao, (10, 100), (10, 100), 2, tab[:5], nblk)
    with pytest.raises(ValueError, match="stride_ao"):
        cm.aodm_fock(v, w, ao, ao, (5, 100), (10, 100), 2, tab, nblk)
    with pytest.raises(ValueError, match="BLKSIZE"):
        cm.aodm_fock(v, w, ao, ao, (10, 100), (10, 100), 2, tab, nblk, blksize=0)
    cm.aodm_fock(v, w, ao, ao, (10, 100), (0, 100), 2, tab, nblk)  # empty: no device needed
    cm.aodm_fock(v, w, ao, ao, (10, 100), (10, 0), 2, tab, nblk)
    cm.aodm_fock(v, w, ao, ao, (10, 100), (10, 100), 0, tab, nblk)
    assert np.all(v == 1)


def test_f32_validation(cm):
    """The f32 forms take the f64 calls' checks (lengths in elements)."""
    a = np.ones((4, 6), np.float32)
    b = np.ones((6, 5), np.float32)
    c = np.zeros((4, 5), np.float32)
    with pytest.raises(ValueError, match="slice too short"):
        cm.matmul_f32(c, a[:2], b, 4, 5, 6, 6, 5, 5, False, False)
    with pytest.raises(ValueError, match="precision"):
        cm.matmul_f32(c, a, b, 4, 5, 6, 6, 5, 5, False, False, precision=9)
    with pytest.raises(TypeError, match="float32"):
        cm.matmul_f32(c.astype(np.float64), a, b, 4, 5, 6, 6, 5, 5, False, False)
    cm.matmul_f32(c, a, b, 0, 5, 6, 6, 5, 5, False, False)  # empty: no device needed
    rho = np.zeros((2, 100), np.float32)
    dms = np.ones((2, 10, 10), np.float32)
    ao = np.ones((10, 100), np.float32)
    tab = np.ones((10, 3), np.uint8)
    with pytest.raises(ValueError, match="slice too short"):
        cm.aodmao2rho_f32(rho, dms[:1], ao, ao, (10, 100), (10, 100), 2, tab, 3)
    with pytest.raises(ValueError, match="BLKSIZE"):
        cm.aodmao2rho_f32(rho, dms, ao, ao, (10, 100), (10, 100), 2, tab, 3, blksize=0)
    cm.aodmao2rho_f32(rho, dms, ao, ao, (10, 100), (10, 100), 0, tab, 3)
    assert np.all(c == 0) and np.all(rho == 0)


def test_bool_mask_is_accepted(cm):
    rho, dms, ao, tab, nblk = _aodm_args()
    with pytest.raises(ValueError, match="slice too short"):
        cm.aodmao2rho_anyway(rho, dms, ao, ao, (10, 100), (10, 100), 2, tab.astype(bool)[:3], nblk)


@pytest.mark.skipif(has_cuda(), reason="checks the no-device path")
def test_no_cpu_fallback_without_device(cm):
    """A valid call on a machine without a GPU must fail loudly, not compute on the CPU."""
    c, a, b = _gemm_args()
    with pytest.raises(cm.CfgmmError) as e:
        cm.matmul_anyway_full(c, a, b, 4, 5, 6, 6, 5, 5, False, False)
    assert e.value.status == -4
    rho, dms, ao, tab, nblk = _aodm_args()
    with pytest.raises(cm.CfgmmError):
        cm.aodmao2rho_anyway(rho, dms, ao, ao, (10, 100), (10, 100), 2, tab, nblk)
    assert np.all(c == 0) and np.all(rho == 0)
    with pytest.raises(cm.CfgmmError):
        cm.aodm_fock(dms, rho, ao, ao, (10, 100), (10, 100), 2, tab, nblk)
    assert np.all(dms == 1)
    with pytest.raises(cm.CfgmmError) as e:
        cm.Server(1 << 30)
    assert e.value.status == -4


def test_noalloc_rejects_what_dev_rejects(cm):
    """The no-allocation contraction runs the argument checks of
    cfgmm_aodmao2rho_dev: overflowing index ranges (stride_ao^2, the set
    stride times nset, the mask extent) get the same status from both, before
    any device is touched."""
    L = ctypes.CDLL(cm.library_path)
    P, S, I = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int
    L.cfgmm_aodmao2rho_dev_noalloc.argtypes = [P, P, P, P, S, S, S, S, S, P, S, S, P]
    L.cfgmm_aodmao2rho_dev_noalloc.restype = I
    L.cfgmm_aodmao2rho_dev.argtypes = [P, P, P, P, S, S, S, S, S, P, S, S, I, P]
    L.cfgmm_aodmao2rho_dev.restype = I
    L.cfgmm_last_error.restype = ctypes.c_char_p
    big = 1 << 33  # stride_ao^2 = 2^66 overflows usize
    fake = 0x1000  # never dereferenced: the checks fail first
    cases = [
        # (stride_ao, stride_grid, nao, ngrid, nset, ldtab, blksize)
        (big, 100, 10, 100, 2, 3, 48),             # stride_ao^2 overflows
        (1 << 31, 100, 10, 100, 1 << 30, 3, 48),  # (nset-1) * stride_ao^2 overflows
        (10, 100, 10, 100, 2, (1 << 63), 48),      # (nao-1) * ldtab overflows
        (10, 50, 10, 100, 2, 3, 48),               # stride_grid < ngrid
        (10, 100, 10, 100, 2, 3, 0),               # BLKSIZE 0
        (10, 100, 1 << 40, 100, 2, 3, 48),         # nao beyond 2^31
    ]
    for sa, sg, nao, ngrid, nset, ldtab, blk in cases:
        args = [fake, fake, fake, fake, sa, sg, nao, ngrid, nset, fake, ldtab, blk]
        rc_dev = L.cfgmm_aodmao2rho_dev(*args, 0, None)
        msg_dev = L.cfgmm_last_error()
        rc_na = L.cfgmm_aodmao2rho_dev_noalloc(*args, None)
        msg_na = L.cfgmm_last_error()
        assert rc_dev == -1, (sa, sg, nao, ngrid, nset, ldtab, blk, msg_dev)
        assert rc_na == rc_dev and msg_na == msg_dev, (msg_na, msg_dev)


def test_arm_wait_timeout_validation(cm):
    """The failure-detection test hook checks its arguments on the host."""
    L = ctypes.CDLL(cm.library_path)
    L.cfgmm_test_arm_wait_timeout.argtypes = [ctypes.c_int, ctypes.c_double]
    L.cfgmm_test_arm_wait_timeout.restype = ctypes.c_int
    assert L.cfgmm_test_arm_wait_timeout(7, 10.0) == -1      # unknown precision
    assert L.cfgmm_test_arm_wait_timeout(0, 0.0) == -1       # below 1 ms
    assert L.cfgmm_test_arm_wait_timeout(1, 5000.0) == -1    # above 2 s
