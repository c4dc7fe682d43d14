"""cfgable-matmul on B200: Python front end of libcfgmm.so.

The functions mirror the reference crate's public API for its two hot paths --
same names, argument order and meaning -- and call the C ABI declared in
include/cfgmm.h through ctypes:

=====================================  ============================================
this module                            reference (paths relative to the crate root)
=====================================  ============================================
``MatmulLoops(...).matmul_loop_parallel_mnk_pack_a``  src/impl_matmul.rs:155-231
``MatmulLoops(...).matmul_loop_macro_mb``             README.md:22-31
``matmul_anyway_full``                                src/impl_matmul.rs:234-248
``MatmulLoops(...).matmul_loop_parallel_mnk_pack_a_non0tab``  src/impl_matmul_non0tab.rs:210-306
``matmul_anyway_full_non0tab``                        src/impl_matmul_non0tab.rs:308-326
``MatmulLoops(...).aodmao2rho_loop_parallel``         src/impl_aodmao2rho.rs:171-244
``aodmao2rho_anyway``                                 src/impl_aodmao2rho.rs:247-261
=====================================  ============================================

Arguments are numpy arrays (host memory; the call is synchronous, like the
reference) or CUDA torch tensors (device memory; the work is enqueued on the
current torch stream).  Outputs are accumulated into.  Where the reference
panics, these functions raise: ``ValueError`` for an argument the reference
would reject by a panic, ``NotImplementedError`` for its ``unimplemented!``,
``RuntimeError`` for a CUDA failure.  There is no CPU fallback: without the
compiled library or a CUDA device every call raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

__all__ = [
    "MatmulLoops", "matmul_anyway_full", "aodmao2rho_anyway", "matmul_ex", "aodmao2rho_ex",
    "matmul_anyway_full_non0tab", "matmul_non0tab_ex",
    "aodmao2rho_noalloc", "AodmPlan", "eval_ao", "mask_ao", "Server",
    "PREC_FP64", "PREC_OZAKI_INT8", "CfgmmError", "lib", "library_path",
]

PREC_FP64 = 0
PREC_OZAKI_INT8 = 1

OK = 0
ERR_INVALID_ARGUMENT = -1
ERR_UNIMPLEMENTED = -2
ERR_CUDA = -3
ERR_NO_DEVICE = -4
ERR_OUT_OF_MEMORY = -5
ERR_TIMEOUT = -6
ERR_BUSY = -7

class _Batch(ctypes.Structure):
    """struct cfgmm_aodm_batch"""
    _fields_ = [("rhos", ctypes.c_void_p), ("ao_lhs", ctypes.c_void_p),
                ("ao_rhs", ctypes.c_void_p), ("tab", ctypes.c_void_p),
                ("stride_grid", ctypes.c_size_t), ("ngrid", ctypes.c_size_t),
                ("ldtab", ctypes.c_size_t), ("nset", ctypes.c_size_t)]


class RequestStats(ctypes.Structure):
    """struct cfgmm_request_stats"""
    _fields_ = [("queue_ms", ctypes.c_double), ("device_ms", ctypes.c_double),
                ("total_ms", ctypes.c_double), ("flops", ctypes.c_double)]


_HERE = os.path.dirname(os.path.abspath(__file__))
library_path = os.path.join(_HERE, "libcfgmm.so")
_lib = None


class CfgmmError(RuntimeError):
    """A CUDA-side failure reported by libcfgmm (status, message)."""

    def __init__(self, status: int, message: str):
        super().__init__(f"libcfgmm status {status}: {message}")
        self.status = status


def lib() -> ctypes.CDLL:
    """Loads libcfgmm.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(library_path):
            raise ImportError(f"{library_path} is missing: run `python cfgable-matmul_b200/build.py`")
        L = ctypes.CDLL(library_path)
        P, S, U8, I = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint8, ctypes.c_int
        gemm_host = [P, S, P, S, P, S, S, S, S, S, S, S, U8, U8]
        for name in ("cfgmm_matmul_loop_parallel_mnk_pack_a", "cfgmm_matmul_anyway_full",
                     "cfgmm_matmul_loop_macro_mb"):
            getattr(L, name).argtypes = gemm_host
            getattr(L, name).restype = I
        L.cfgmm_matmul_ex.argtypes = gemm_host + [I]
        L.cfgmm_matmul_ex.restype = I
        L.cfgmm_matmul_dev.argtypes = [P, P, P, S, S, S, S, S, S, U8, U8, I, P]
        L.cfgmm_matmul_dev.restype = I
        mask_host = gemm_host + [P, S, S]
        L.cfgmm_matmul_anyway_full_non0tab.argtypes = mask_host
        L.cfgmm_matmul_anyway_full_non0tab.restype = I
        L.cfgmm_matmul_loop_parallel_mnk_pack_a_non0tab.argtypes = mask_host + [S]
        L.cfgmm_matmul_loop_parallel_mnk_pack_a_non0tab.restype = I
        L.cfgmm_matmul_non0tab_ex.argtypes = mask_host + [S, I]
        L.cfgmm_matmul_non0tab_ex.restype = I
        L.cfgmm_matmul_non0tab_dev.argtypes = [P, P, P, S, S, S, S, S, S, U8, U8, P, S, S, I, P]
        L.cfgmm_matmul_non0tab_dev.restype = I
        L.cfgmm_matmul_dev_timed.argtypes = [P, P, P, S, S, S, S, S, S, U8, U8, I, P,
                                             ctypes.POINTER(P), I]
        L.cfgmm_matmul_dev_timed.restype = I
        L.cfgmm_split_moduli.argtypes = [S]
        L.cfgmm_split_moduli.restype = I
        L.cfgmm_device_check.restype = I
        aodm_host = [P, S, P, S, P, S, P, S, S, S, S, S, S, P, S, S]
        L.cfgmm_aodmao2rho_anyway.argtypes = aodm_host
        L.cfgmm_aodmao2rho_anyway.restype = I
        L.cfgmm_aodmao2rho_loop_parallel.argtypes = aodm_host + [S]
        L.cfgmm_aodmao2rho_loop_parallel.restype = I
        L.cfgmm_aodmao2rho_ex.argtypes = aodm_host + [S, I]
        L.cfgmm_aodmao2rho_ex.restype = I
        L.cfgmm_aodmao2rho_dev.argtypes = [P, P, P, P, S, S, S, S, S, P, S, S, I, P]
        L.cfgmm_aodmao2rho_dev.restype = I
        L.cfgmm_status_string.argtypes = [I]
        L.cfgmm_status_string.restype = ctypes.c_char_p
        L.cfgmm_last_error.restype = ctypes.c_char_p
        L.cfgmm_version.restype = I
        L.cfgmm_release_workspace.restype = I
        L.cfgmm_aodmao2rho_dev_noalloc.argtypes = [P, P, P, P, S, S, S, S, S, P, S, S, P]
        L.cfgmm_aodmao2rho_dev_noalloc.restype = I
        L.cfgmm_aodm_fock.argtypes = aodm_host + [S]
        L.cfgmm_aodm_fock.restype = I
        L.cfgmm_aodm_fock_dev.argtypes = [P, P, P, P, S, S, S, S, S, P, S, S, P]
        L.cfgmm_aodm_fock_dev.restype = I
        L.cfgmm_matmul_f32.argtypes = [P, S, P, S, P, S] + [S] * 6 + [U8, U8, I]
        L.cfgmm_matmul_f32.restype = I
        L.cfgmm_matmul_f32_dev.argtypes = [P, P, P] + [S] * 6 + [U8, U8, I, P]
        L.cfgmm_matmul_f32_dev.restype = I
        L.cfgmm_aodmao2rho_f32.argtypes = aodm_host + [S, I]
        L.cfgmm_aodmao2rho_f32.restype = I
        L.cfgmm_aodmao2rho_f32_dev.argtypes = [P, P, P, P, S, S, S, S, S, P, S, S, I, P]
        L.cfgmm_aodmao2rho_f32_dev.restype = I
        L.cfgmm_aodm_plan_create.argtypes = [ctypes.POINTER(P), ctypes.POINTER(_Batch), S, P, S,
                                             S, S, S, I, I, P]
        L.cfgmm_aodm_plan_create.restype = I
        L.cfgmm_aodm_plan_run.argtypes = [P, P]
        L.cfgmm_aodm_plan_run.restype = I
        L.cfgmm_aodm_plan_info.argtypes = [P]
        L.cfgmm_aodm_plan_info.restype = ctypes.c_char_p
        L.cfgmm_aodm_plan_destroy.argtypes = [P]
        L.cfgmm_aodm_plan_destroy.restype = I
        L.cfgmm_eval_ao_dev.argtypes = [P, S, P, S, P, P, P, P, P, S, P, S, P]
        L.cfgmm_eval_ao_dev.restype = I
        L.cfgmm_mask_ao_dev.argtypes = [P, S, S, P, P, S, P, ctypes.c_double, P, S, S, P]
        L.cfgmm_mask_ao_dev.restype = I
        U64 = ctypes.c_uint64
        L.cfgmm_server_create.argtypes = [ctypes.POINTER(P), S, I, I, S]
        L.cfgmm_server_create.restype = I
        L.cfgmm_server_destroy.argtypes = [P]
        L.cfgmm_server_destroy.restype = I
        L.cfgmm_server_open.argtypes = [P, P, P, P, S, S, S, S, I, ctypes.POINTER(U64)]
        L.cfgmm_server_open.restype = I
        L.cfgmm_server_open_shells.argtypes = [P, P, S, P, P, P, P, S, ctypes.c_double, S,
                                               ctypes.POINTER(U64)]
        L.cfgmm_server_open_shells.restype = I
        L.cfgmm_server_close.argtypes = [P, U64]
        L.cfgmm_server_close.restype = I
        L.cfgmm_server_submit.argtypes = [P, U64, P, S, P, ctypes.POINTER(U64)]
        L.cfgmm_server_submit.restype = I
        L.cfgmm_server_submit_dev.argtypes = [P, U64, P, S, P, P, ctypes.POINTER(U64)]
        L.cfgmm_server_submit_dev.restype = I
        L.cfgmm_server_wait.argtypes = [P, U64, ctypes.c_double, ctypes.POINTER(RequestStats)]
        L.cfgmm_server_wait.restype = I
        L.cfgmm_server_stats.argtypes = [P]
        L.cfgmm_server_stats.restype = ctypes.c_char_p
        _lib = L
    return _lib


def _raise(rc: int) -> None:
    if rc == OK:
        return
    msg = lib().cfgmm_last_error().decode(errors="replace") or lib().cfgmm_status_string(rc).decode()
    if rc == ERR_INVALID_ARGUMENT:
        raise ValueError(msg)
    if rc == ERR_UNIMPLEMENTED:
        raise NotImplementedError(msg)
    raise CfgmmError(rc, msg)


def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


def _host(x, dtype, writable=False):
    """(pointer, length) of a C-contiguous numpy array of `dtype`."""
    if not isinstance(x, np.ndarray):
        raise TypeError("expected a numpy array or a CUDA torch tensor")
    if x.dtype != dtype:
        raise TypeError(f"expected dtype {np.dtype(dtype).name}, got {x.dtype}")
    if not x.flags.c_contiguous:
        raise ValueError("arrays must be C-contiguous (a Rust slice is contiguous)")
    if writable and not x.flags.writeable:
        raise ValueError("output array is read-only")
    return x.ctypes.data, x.size


def _dev(x, dtype_name):
    if not x.is_cuda or not x.is_contiguous():
        raise ValueError("device tensors must be contiguous CUDA tensors")
    if str(x.dtype) != dtype_name:
        raise TypeError(f"expected {dtype_name}, got {x.dtype}")
    return x.data_ptr()


def _stream_ptr():
    import torch
    return torch.cuda.current_stream().cuda_stream


def _as_tab(tab):
    if isinstance(tab, np.ndarray) and tab.dtype == np.bool_:
        return tab.view(np.uint8)
    if _is_torch(tab) and str(tab.dtype) == "torch.bool":
        return tab.view(dtype=__import__("torch").uint8)
    return tab


def matmul_ex(c, a, b, m, n, k, lda, ldb, ldc, transa, transb, precision=PREC_FP64) -> None:
    """C += op(A) op(B) with an explicit arithmetic (PREC_FP64 / PREC_OZAKI_INT8)."""
    if _is_torch(c):
        rc = lib().cfgmm_matmul_dev(_dev(c, "torch.float64"), _dev(a, "torch.float64"),
                                    _dev(b, "torch.float64"), m, n, k, lda, ldb, ldc,
                                    int(bool(transa)), int(bool(transb)), precision, _stream_ptr())
        return _raise(rc)
    pc, lc = _host(c, np.float64, True)
    pa, la = _host(a, np.float64)
    pb, lb = _host(b, np.float64)
    _raise(lib().cfgmm_matmul_ex(pc, lc, pa, la, pb, lb, m, n, k, lda, ldb, ldc,
                                 int(bool(transa)), int(bool(transb)), precision))


def matmul_anyway_full(c, a, b, m, n, k, lda, ldb, ldc, transa, transb) -> None:
    """C[i*ldc+j] += sum_p opA(i,p) opB(p,j) (src/impl_matmul.rs:234-248)."""
    if _is_torch(c):
        return matmul_ex(c, a, b, m, n, k, lda, ldb, ldc, transa, transb)
    pc, lc = _host(c, np.float64, True)
    pa, la = _host(a, np.float64)
    pb, lb = _host(b, np.float64)
    _raise(lib().cfgmm_matmul_anyway_full(pc, lc, pa, la, pb, lb, m, n, k, lda, ldb, ldc,
                                          int(bool(transa)), int(bool(transb))))


def matmul_non0tab_ex(c, a, b, m, n, k, lda, ldb, ldc, transa, transb, tab, ldtab, blksize=48,
                      precision=PREC_FP64) -> None:
    """Masked GEMM C[i,j] += sum_{p: tab[p, j/BLK]} opA(i,p) B[p,j] with an explicit
    BLKSIZE and arithmetic; transb raises NotImplementedError as the reference panics."""
    tab = _as_tab(tab)
    if _is_torch(c):
        rc = lib().cfgmm_matmul_non0tab_dev(
            _dev(c, "torch.float64"), _dev(a, "torch.float64"), _dev(b, "torch.float64"), m, n, k,
            lda, ldb, ldc, int(bool(transa)), int(bool(transb)), _dev(tab, "torch.uint8"), ldtab,
            blksize, precision, _stream_ptr())
        return _raise(rc)
    pc, lc = _host(c, np.float64, True)
    pa, la = _host(a, np.float64)
    pb, lb = _host(b, np.float64)
    pt, lt = _host(tab, np.uint8)
    _raise(lib().cfgmm_matmul_non0tab_ex(pc, lc, pa, la, pb, lb, m, n, k, lda, ldb, ldc,
                                         int(bool(transa)), int(bool(transb)), pt, lt, ldtab,
                                         blksize, precision))


def matmul_anyway_full_non0tab(c, a, b, m, n, k, lda, ldb, ldc, transa, transb, tab,
                               ldtab) -> None:
    """Masked GEMM with BLKSIZE 48 (src/impl_matmul_non0tab.rs:308-326)."""
    if _is_torch(c):
        return matmul_non0tab_ex(c, a, b, m, n, k, lda, ldb, ldc, transa, transb, tab, ldtab, 48)
    pc, lc = _host(c, np.float64, True)
    pa, la = _host(a, np.float64)
    pb, lb = _host(b, np.float64)
    pt, lt = _host(_as_tab(tab), np.uint8)
    _raise(lib().cfgmm_matmul_anyway_full_non0tab(pc, lc, pa, la, pb, lb, m, n, k, lda, ldb, ldc,
                                                  int(bool(transa)), int(bool(transb)), pt, lt,
                                                  ldtab))


def aodmao2rho_ex(rhos, dms, ao_lhs, ao_rhs, strides, shape, nset, tab, ldtab, blksize=48,
                  precision=PREC_FP64) -> None:
    """The masked AO-DM-AO contraction with an explicit BLKSIZE and arithmetic."""
    stride_ao, stride_grid = strides
    nao, ngrid = shape
    tab = _as_tab(tab)
    if _is_torch(rhos):
        rc = lib().cfgmm_aodmao2rho_dev(
            _dev(rhos, "torch.float64"), _dev(dms, "torch.float64"), _dev(ao_lhs, "torch.float64"),
            _dev(ao_rhs, "torch.float64"), stride_ao, stride_grid, nao, ngrid, nset,
            _dev(tab, "torch.uint8"), ldtab, blksize, precision, _stream_ptr())
        return _raise(rc)
    pr, lr = _host(rhos, np.float64, True)
    pd, ld = _host(dms, np.float64)
    pl, ll = _host(ao_lhs, np.float64)
    pq, lq = _host(ao_rhs, np.float64)
    pt, lt = _host(tab, np.uint8)
    _raise(lib().cfgmm_aodmao2rho_ex(pr, lr, pd, ld, pl, ll, pq, lq, stride_ao, stride_grid, nao,
                                     ngrid, nset, pt, lt, ldtab, blksize, precision))


def aodmao2rho_anyway(rhos, dms, ao_lhs, ao_rhs, strides, shape, nset, tab, ldtab) -> None:
    """rho[s,g] += sum_{u,v} ao_lhs[u,g] D_s[u,v] ao_rhs[v,g] over the AOs active in
    g's block of 48 points (src/impl_aodmao2rho.rs:247-261)."""
    if _is_torch(rhos):
        return aodmao2rho_ex(rhos, dms, ao_lhs, ao_rhs, strides, shape, nset, tab, ldtab, 48)
    stride_ao, stride_grid = strides
    nao, ngrid = shape
    pr, lr = _host(rhos, np.float64, True)
    pd, ld = _host(dms, np.float64)
    pl, ll = _host(ao_lhs, np.float64)
    pq, lq = _host(ao_rhs, np.float64)
    pt, lt = _host(_as_tab(tab), np.uint8)
    _raise(lib().cfgmm_aodmao2rho_anyway(pr, lr, pd, ld, pl, ll, pq, lq, stride_ao, stride_grid,
                                         nao, ngrid, nset, pt, lt, ldtab))


def aodmao2rho_noalloc(rhos, dms, ao_lhs, ao_rhs, strides, shape, nset, tab, ldtab,
                       blksize=48) -> None:
    """The FP64 contraction on device tensors with no allocation: scratch lives
    in a fixed static device array, so overlapping calls race (see cfgmm.h)."""
    stride_ao, stride_grid = strides
    nao, ngrid = shape
    tab = _as_tab(tab)
    _raise(lib().cfgmm_aodmao2rho_dev_noalloc(
        _dev(rhos, "torch.float64"), _dev(dms, "torch.float64"), _dev(ao_lhs, "torch.float64"),
        _dev(ao_rhs, "torch.float64"), stride_ao, stride_grid, nao, ngrid, nset,
        _dev(tab, "torch.uint8"), ldtab, blksize, _stream_ptr()))


def matmul_f32(c, a, b, m, n, k, lda, ldb, ldc, transa, transb, precision=PREC_FP64) -> None:
    """C += op(A) op(B) on f32 data (MatmulLoops<f32>; the reference implements
    only f64, src/structs.rs:19-20): f64 arithmetic inside, one rounding to f32.
    numpy float32 arrays (synchronous) or float32 CUDA tensors (current stream)."""
    if _is_torch(c):
        return _raise(lib().cfgmm_matmul_f32_dev(
            _dev(c, "torch.float32"), _dev(a, "torch.float32"), _dev(b, "torch.float32"),
            m, n, k, lda, ldb, ldc, int(transa), int(transb), precision, _stream_ptr()))
    pc, lc = _host(c, np.float32, True)
    pa, la = _host(a, np.float32)
    pb, lb = _host(b, np.float32)
    _raise(lib().cfgmm_matmul_f32(pc, lc, pa, la, pb, lb, m, n, k, lda, ldb, ldc, int(transa),
                                  int(transb), precision))


def aodmao2rho_f32(rhos, dms, ao_lhs, ao_rhs, strides, shape, nset, tab, ldtab, blksize=48,
                   precision=PREC_FP64) -> None:
    """The masked AO-DM-AO contraction on f32 data, f64 arithmetic inside and
    one rounding of rho to f32; arguments as aodmao2rho_ex."""
    stride_ao, stride_grid = strides
    nao, ngrid = shape
    tab = _as_tab(tab)
    if _is_torch(rhos):
        return _raise(lib().cfgmm_aodmao2rho_f32_dev(
            _dev(rhos, "torch.float32"), _dev(dms, "torch.float32"), _dev(ao_lhs, "torch.float32"),
            _dev(ao_rhs, "torch.float32"), stride_ao, stride_grid, nao, ngrid, nset,
            _dev(tab, "torch.uint8"), ldtab, blksize, precision, _stream_ptr()))
    pr, lr = _host(rhos, np.float32, True)
    pd, ld = _host(dms, np.float32)
    pl, ll = _host(ao_lhs, np.float32)
    pq, lq = _host(ao_rhs, np.float32)
    pt, lt = _host(tab, np.uint8)
    _raise(lib().cfgmm_aodmao2rho_f32(pr, lr, pd, ld, pl, ll, pq, lq, stride_ao, stride_grid, nao,
                                      ngrid, nset, pt, lt, ldtab, blksize, precision))


def aodm_fock(vs, ws, ao_lhs, ao_rhs, strides, shape, nset, tab, ldtab, blksize=48) -> None:
    """The Fock-build contraction, the transpose of the AO-DM-AO one on the same
    layouts and mask: V_s[u,v] += sum_g ao_lhs[u,g] w_s[g] ao_rhs[v,g] over the
    points g whose block has both u and v active.  ``vs`` (nset, stride_ao,
    stride_ao) takes D's place, ``ws`` (nset, stride_grid) rho's.  FP64 on the
    tensor cores; numpy arrays go through host buffers, CUDA tensors run on the
    current stream.  No counterpart in the reference."""
    stride_ao, stride_grid = strides
    nao, ngrid = shape
    tab = _as_tab(tab)
    if _is_torch(vs):
        return _raise(lib().cfgmm_aodm_fock_dev(
            _dev(vs, "torch.float64"), _dev(ws, "torch.float64"), _dev(ao_lhs, "torch.float64"),
            _dev(ao_rhs, "torch.float64"), stride_ao, stride_grid, nao, ngrid, nset,
            _dev(tab, "torch.uint8"), ldtab, blksize, _stream_ptr()))
    pv, lv = _host(vs, np.float64, True)
    pw, lw = _host(ws, np.float64)
    pl, ll = _host(ao_lhs, np.float64)
    pq, lq = _host(ao_rhs, np.float64)
    pt, lt = _host(tab, np.uint8)
    _raise(lib().cfgmm_aodm_fock(pv, lv, pw, lw, pl, ll, pq, lq, stride_ao, stride_grid, nao,
                                 ngrid, nset, pt, lt, ldtab, blksize))


class AodmPlan:
    """Many grid batches of one molecule contracted by one persistent launch.

    ``batches`` is a list of ``(rhos, ao_lhs, ao_rhs, tab, nset)`` CUDA tensors
    (rhos (>=nset, ngrid), phi (nao, ngrid), tab (nao, nblk) uint8); ``dms`` is
    (nset_max, nao, nao).  The tensors are referenced, not copied: phi and the
    masks must stay unchanged while the plan lives, the contents of ``dms`` may
    change between runs.  ``run()`` accumulates into every batch's rho on the
    current stream.  No counterpart in the reference, whose callers loop over
    grid batches (src/impl_matmul.rs:354-355 is the grid loop of its driver)."""

    def __init__(self, batches, dms, blksize=64, precision=PREC_FP64, graph=True, tune=True):
        self._keep = (list(batches), dms)
        nao = dms.shape[-1]
        arr = (_Batch * max(1, len(batches)))()
        for i, (rhos, ao_lhs, ao_rhs, tab, nset) in enumerate(batches):
            tab = _as_tab(tab)
            arr[i] = _Batch(_dev(rhos, "torch.float64"), _dev(ao_lhs, "torch.float64"),
                            _dev(ao_rhs, "torch.float64"), _dev(tab, "torch.uint8"),
                            ao_lhs.shape[1], ao_lhs.shape[1], tab.shape[1], nset)
        flags = (0 if graph else 1) | (0 if tune else 2)
        h = ctypes.c_void_p()
        _raise(lib().cfgmm_aodm_plan_create(ctypes.byref(h), arr, len(batches),
                                            _dev(dms, "torch.float64"), nao, nao, dms.shape[0],
                                            blksize, precision, flags, _stream_ptr()))
        self._h = h

    def run(self) -> None:
        _raise(lib().cfgmm_aodm_plan_run(self._h, _stream_ptr()))

    def info(self) -> dict:
        import json
        return json.loads(lib().cfgmm_aodm_plan_info(self._h).decode())

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().cfgmm_aodm_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def eval_ao(ao, points, shell_xyz, shell_l, shell_alpha, shell_norm, shell_row,
            shell_block_max=None, blksize=64) -> None:
    """phi (nao, ngrid) of Gaussian shells (l <= 3, real solid harmonics) on the
    points (ngrid, 3), all CUDA tensors; optionally max|phi| per (shell, block)."""
    ngrid = points.shape[0]
    _raise(lib().cfgmm_eval_ao_dev(
        _dev(ao, "torch.float64"), ao.shape[1], _dev(points, "torch.float64"), ngrid,
        _dev(shell_xyz, "torch.float64"), _dev(shell_l, "torch.int32"),
        _dev(shell_alpha, "torch.float64"), _dev(shell_norm, "torch.float64"),
        _dev(shell_row, "torch.int32"), shell_l.shape[0],
        None if shell_block_max is None else _dev(shell_block_max, "torch.float64"), blksize,
        _stream_ptr()))


def mask_ao(ao, ngrid, shell_l, shell_row, shell_block_max, threshold, tab, blksize=64) -> None:
    """tab[row, b] = shell_block_max[shell(row), b] > threshold; phi zeroed where 0."""
    _raise(lib().cfgmm_mask_ao_dev(
        _dev(ao, "torch.float64"), ao.shape[1], ngrid, _dev(shell_l, "torch.int32"),
        _dev(shell_row, "torch.int32"), shell_l.shape[0], _dev(shell_block_max, "torch.float64"),
        float(threshold), _dev(tab, "torch.uint8"), tab.shape[1], blksize, _stream_ptr()))


class Server:
    """Density requests from many molecules with continuous batching under an
    HBM budget (cfgmm_server_*).  No counterpart in the reference.

    ``open(ao, tab, nset_max)`` takes numpy arrays (uploaded on admission;
    keep them alive until ``close``) or CUDA tensors (used in place);
    ``open_shells(points, shell_xyz, shell_l, shell_alpha, shell_norm,
    density, nset_max)`` evaluates phi and the mask on the device.
    ``submit(mol, dms, rho)`` returns a ticket at once (dms copied, rho
    written on completion); ``wait(ticket)`` returns the request's
    (queue_ms, device_ms, total_ms, flops)."""

    def __init__(self, hbm_budget, nslots=4, precision=PREC_FP64, blksize=64):
        h = ctypes.c_void_p()
        _raise(lib().cfgmm_server_create(ctypes.byref(h), int(hbm_budget), nslots, precision,
                                         blksize))
        self._h = h
        self._keep = {}
        self.blksize = blksize

    def open(self, ao_lhs, tab, nset_max, ao_rhs=None):
        tab = _as_tab(tab)
        nao, ngrid = ao_lhs.shape
        mol = ctypes.c_uint64()
        if _is_torch(ao_lhs):
            ptrs = (_dev(ao_lhs, "torch.float64"),
                    None if ao_rhs is None else _dev(ao_rhs, "torch.float64"),
                    _dev(tab, "torch.uint8"))
            dev = 1
        else:
            ptrs = (_host(ao_lhs, np.float64)[0],
                    None if ao_rhs is None else _host(ao_rhs, np.float64)[0],
                    _host(tab, np.uint8)[0])
            dev = 0
        _raise(lib().cfgmm_server_open(self._h, ptrs[0], ptrs[1], ptrs[2], nao, ngrid,
                                       tab.shape[1], nset_max, dev, ctypes.byref(mol)))
        self._keep[mol.value] = (ao_lhs, ao_rhs, tab)
        return mol.value

    def open_shells(self, points, shell_xyz, shell_l, shell_alpha, shell_norm, density,
                    nset_max):
        arrs = [np.ascontiguousarray(points, np.float64), np.ascontiguousarray(shell_xyz, np.float64),
                np.ascontiguousarray(shell_l, np.int32), np.ascontiguousarray(shell_alpha, np.float64),
                np.ascontiguousarray(shell_norm, np.float64)]
        mol = ctypes.c_uint64()
        _raise(lib().cfgmm_server_open_shells(self._h, arrs[0].ctypes.data, len(arrs[0]),
                                              arrs[1].ctypes.data, arrs[2].ctypes.data,
                                              arrs[3].ctypes.data, arrs[4].ctypes.data,
                                              len(arrs[2]), float(density), nset_max,
                                              ctypes.byref(mol)))
        return mol.value

    def close(self, mol) -> None:
        _raise(lib().cfgmm_server_close(self._h, mol))
        self._keep.pop(mol, None)

    def submit(self, mol, dms, rho) -> int:
        """Host numpy arrays: D copied now, rho written on completion.  CUDA
        tensors (cfgmm_server_submit_dev): D read once the current stream's
        work so far is done, rho overwritten on the device; both must stay
        untouched until the ticket is waited for."""
        t = ctypes.c_uint64()
        if _is_torch(dms) or _is_torch(rho):
            if not (_is_torch(dms) and _is_torch(rho)) or dms.dim() != 3 or rho.dim() != 2 \
                    or rho.shape[0] != dms.shape[0]:
                raise ValueError("device submit: dms (nset, nao, nao) and rho (nset, ngrid), "
                                 "both CUDA tensors")
            _raise(lib().cfgmm_server_submit_dev(self._h, mol, _dev(dms, "torch.float64"),
                                                 dms.shape[0], _dev(rho, "torch.float64"),
                                                 _stream_ptr(), ctypes.byref(t)))
            self._keep[("rho", t.value)] = (dms, rho)
            return t.value
        pd, _ = _host(dms, np.float64)
        pr, _ = _host(rho, np.float64, True)
        _raise(lib().cfgmm_server_submit(self._h, mol, pd, dms.shape[0], pr, ctypes.byref(t)))
        self._keep[("rho", t.value)] = rho
        return t.value

    def wait(self, ticket, timeout=-1.0):
        st = RequestStats()
        rc = lib().cfgmm_server_wait(self._h, ticket, float(timeout), ctypes.byref(st))
        if rc != ERR_TIMEOUT:  # a timed-out request still owns its rho buffer
            self._keep.pop(("rho", ticket), None)
        _raise(rc)
        return st.queue_ms, st.device_ms, st.total_ms, st.flops

    def stats(self) -> dict:
        import json
        return json.loads(lib().cfgmm_server_stats(self._h).decode())

    def shutdown(self) -> None:
        if getattr(self, "_h", None):
            lib().cfgmm_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.shutdown()
        except Exception:
            pass


class MatmulLoops:
    """Mirror of ``MatmulLoops<T, MC, KC, NC, MR, NR_LANE, LANE>`` (src/structs.rs:15).

    The const generics select CPU cache and register blocking in the
    reference; on the GPU the library picks its own tiles, so they are kept
    only for signature compatibility.  ``dtype`` must be float64: the
    reference implements the micro-kernel for f64 only (src/structs.rs:19-20).
    """

    def __init__(self, dtype=np.float64, MC=252, KC=512, NC=240, MR=14, NR_LANE=2, LANE=8, MB=None):
        if np.dtype(dtype) != np.float64:
            raise TypeError("MatmulLoops is implemented for f64 only")
        self.tuning = dict(MC=MC, KC=KC, NC=NC, MR=MR, NR_LANE=NR_LANE, LANE=LANE, MB=MB)

    def matmul_loop_parallel_mnk_pack_a(self, c, a, b, m, n, k, lda, ldb, ldc, transa, transb):
        """src/impl_matmul.rs:155-231"""
        if _is_torch(c):
            return matmul_ex(c, a, b, m, n, k, lda, ldb, ldc, transa, transb)
        pc, lc = _host(c, np.float64, True)
        pa, la = _host(a, np.float64)
        pb, lb = _host(b, np.float64)
        _raise(lib().cfgmm_matmul_loop_parallel_mnk_pack_a(pc, lc, pa, la, pb, lb, m, n, k, lda,
                                                           ldb, ldc, int(bool(transa)),
                                                           int(bool(transb))))

    def matmul_loop_macro_mb(self, c, a, b, m, n, k, lda, ldb, ldc, transa, transb):
        """README.md:22-31 (documented there, absent from the crate's sources)."""
        if _is_torch(c):
            return matmul_ex(c, a, b, m, n, k, lda, ldb, ldc, transa, transb)
        pc, lc = _host(c, np.float64, True)
        pa, la = _host(a, np.float64)
        pb, lb = _host(b, np.float64)
        _raise(lib().cfgmm_matmul_loop_macro_mb(pc, lc, pa, la, pb, lb, m, n, k, lda, ldb, ldc,
                                                int(bool(transa)), int(bool(transb))))

    def matmul_loop_parallel_mnk_pack_a_non0tab(self, c, a, b, m, n, k, lda, ldb, ldc, transa,
                                                transb, tab, ldtab, BLKSIZE=48):
        """src/impl_matmul_non0tab.rs:210-306; BLKSIZE is the const generic."""
        if _is_torch(c):
            return matmul_non0tab_ex(c, a, b, m, n, k, lda, ldb, ldc, transa, transb, tab, ldtab,
                                     BLKSIZE)
        pc, lc = _host(c, np.float64, True)
        pa, la = _host(a, np.float64)
        pb, lb = _host(b, np.float64)
        pt, lt = _host(_as_tab(tab), np.uint8)
        _raise(lib().cfgmm_matmul_loop_parallel_mnk_pack_a_non0tab(
            pc, lc, pa, la, pb, lb, m, n, k, lda, ldb, ldc, int(bool(transa)), int(bool(transb)),
            pt, lt, ldtab, BLKSIZE))

    def aodmao2rho_loop_parallel(self, rhos, dms, ao_lhs, ao_rhs, strides, shape, nset, tab,
                                 ldtab, BLKSIZE=48):
        """src/impl_aodmao2rho.rs:171-244; BLKSIZE is the const generic."""
        if _is_torch(rhos):
            return aodmao2rho_ex(rhos, dms, ao_lhs, ao_rhs, strides, shape, nset, tab, ldtab,
                                 BLKSIZE)
        stride_ao, stride_grid = strides
        nao, ngrid = shape
        pr, lr = _host(rhos, np.float64, True)
        pd, ld = _host(dms, np.float64)
        pl, ll = _host(ao_lhs, np.float64)
        pq, lq = _host(ao_rhs, np.float64)
        pt, lt = _host(_as_tab(tab), np.uint8)
        _raise(lib().cfgmm_aodmao2rho_loop_parallel(pr, lr, pd, ld, pl, ll, pq, lq, stride_ao,
                                                    stride_grid, nao, ngrid, nset, pt, lt, ldtab,
                                                    BLKSIZE))
