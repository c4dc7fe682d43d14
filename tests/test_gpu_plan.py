"""GPU tests of batched AO-DM-AO plans (cfgmm_aodm_plan_*).

A plan contracts many grid batches of one molecule in one persistent launch.
Its result must equal, batch by batch, the single-call contraction (which is
itself pinned to the oracle), with and without the CUDA graph and the
autotuner; runs accumulate; new density-matrix contents are picked up by the
captured graph; the autotuner's choice is cached on disk and reused.
"""
import json
import os

import numpy as np
import pytest

from conftest import normwise

pytestmark = pytest.mark.gpu
TOL = 1e-13


def _batches(wl, torch, seed, nbatch, nao=200, nset_max=3, blk=64):
    """Uneven ragged batches (ngrid 1..700, densities 0..1) of random phi."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(nbatch):
        ngrid = int(rng.integers(1, 700))
        nblk = -(-ngrid // blk)
        dens = [0.0, 1.0, rng.uniform(0.05, 0.6)][i % 3] if i < 6 else rng.uniform(0.05, 0.6)
        tab = (rng.random((nao, nblk)) < dens).astype(np.uint8)
        lhs = rng.standard_normal((nao, ngrid))
        rhs = rng.standard_normal((nao, ngrid))
        m = wl.expand_mask(tab, ngrid, blk)
        lhs[~m] = 0.0
        rhs[~m] = 0.0
        nset = int(rng.integers(1, nset_max + 1))
        rho0 = rng.standard_normal((nset, ngrid))
        out.append(dict(lhs=lhs, rhs=rhs, tab=tab, nset=nset, rho0=rho0, ngrid=ngrid))
    dms = rng.standard_normal((nset_max, nao, nao))
    return out, dms


def _device(torch, bs, dms):
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    dev = [(t(b["rho0"]), t(b["lhs"]), t(b["rhs"]), t(b["tab"]), b["nset"]) for b in bs]
    return dev, t(dms)


def _single(cm, torch, b, dms, blk, precision=0):
    nao, ngrid = b["lhs"].shape
    rho = b["rho0"].copy()
    cm.aodmao2rho_ex(rho, np.ascontiguousarray(dms[: b["nset"]]), b["lhs"], b["rhs"],
                     (nao, ngrid), (nao, ngrid), b["nset"], b["tab"], b["tab"].shape[1], blk,
                     precision)
    return rho


@pytest.mark.parametrize("graph,tune", [(True, True), (False, False), (True, False)])
def test_plan_equals_single_calls(cm, wl, tmp_path, monkeypatch, graph, tune):
    import torch
    monkeypatch.setenv("CFGMM_AUTOTUNE_CACHE", str(tmp_path / "tune.txt"))
    bs, dms = _batches(wl, torch, 1, 23)
    dev, ddms = _device(torch, bs, dms)
    plan = cm.AodmPlan(dev, ddms, blksize=64, graph=graph, tune=tune)
    plan.run()
    torch.cuda.synchronize()
    info = plan.info()
    assert info["batches"] == 23 and info["graph"] is graph
    for b, d in zip(bs, dev):
        ref = _single(cm, torch, b, dms, 64)
        assert normwise(d[0].cpu().numpy(), ref) < TOL
    plan.close()


def test_plan_runs_accumulate_and_follow_dms(cm, wl):
    import torch
    bs, dms = _batches(wl, torch, 2, 9, nao=130)
    for b in bs:
        b["rho0"][:] = 0.0
    dev, ddms = _device(torch, bs, dms)
    plan = cm.AodmPlan(dev, ddms, blksize=64, tune=False)
    plan.run()
    plan.run()
    torch.cuda.synchronize()
    for b, d in zip(bs, dev):
        ref = _single(cm, torch, b, dms, 64)
        assert normwise(d[0].cpu().numpy(), 2.0 * ref) < TOL
    # new DM contents (an SCF step): the captured graph reads them
    dms2 = -0.5 * dms + 1.0
    ddms.copy_(torch.from_numpy(dms2))
    for d in dev:
        d[0].zero_()
    plan.run()
    torch.cuda.synchronize()
    for b, d in zip(bs, dev):
        ref = _single(cm, torch, b, dms2, 64)
        assert normwise(d[0].cpu().numpy(), ref) < TOL
    plan.close()


def test_plan_other_block_sizes(cm, wl):
    import torch
    for blk in (48, 128, 200):
        bs, dms = _batches(wl, torch, blk, 7, nao=97, blk=blk)
        dev, ddms = _device(torch, bs, dms)
        plan = cm.AodmPlan(dev, ddms, blksize=blk, tune=False)
        plan.run()
        torch.cuda.synchronize()
        for b, d in zip(bs, dev):
            ref = _single(cm, torch, b, dms, blk)
            assert normwise(d[0].cpu().numpy(), ref) < TOL
        plan.close()


def test_autotune_cache(cm, wl, tmp_path, monkeypatch):
    import torch
    path = tmp_path / "sub" / "tune.txt"
    monkeypatch.setenv("CFGMM_AUTOTUNE_CACHE", str(path))
    bs, dms = _batches(wl, torch, 3, 12)
    dev, ddms = _device(torch, bs, dms)
    p1 = cm.AodmPlan(dev, ddms, blksize=64)
    i1 = p1.info()
    # ns 1..3 for each form: the pipelined kernel (tk 0) and form 3 at tk 32, 16
    assert isinstance(i1["tuning"], list) and len(i1["tuning"]) == 9
    assert sorted({t["tk"] for t in i1["tuning"]}) == [0, 16, 32]
    assert min(t["ms"] for t in i1["tuning"]) > 0
    lines = path.read_text().split()
    assert lines[0] == i1["key"]
    p2 = cm.AodmPlan(dev, ddms, blksize=64)
    i2 = p2.info()
    assert i2["tuning"] == "cache" and i2["config"] == i1["config"]
    p1.close()
    p2.close()


@pytest.mark.parametrize("form", ["row", "pair"])
@pytest.mark.parametrize("graph,tune", [(True, True), (False, False)])
def test_split_plan_equals_single_split_calls(cm, wl, tmp_path, monkeypatch, graph, tune, form):
    """The split plan keeps phi digits from creation and rebuilds D digits per
    run; its arithmetic is the single call's, so results match bit for bit,
    and stay within 1e-12 of FP64."""
    import torch
    monkeypatch.setenv("CFGMM_AUTOTUNE_CACHE", str(tmp_path / "tune.txt"))
    monkeypatch.setenv("CFGMM_SPLIT_FORM", form)
    bs, dms = _batches(wl, torch, 11, 17)
    dev, ddms = _device(torch, bs, dms)
    plan = cm.AodmPlan(dev, ddms, blksize=64, precision=cm.PREC_OZAKI_INT8, graph=graph, tune=tune)
    info = plan.info()
    assert info["precision"] == "split" and info["graph"] is graph
    if tune:
        stages = [t["stages"] for t in info["tuning"]]
        assert stages in ([3, 4, 5], [3])  # row form: three depths; pair form: fixed
        assert min(t["ms"] for t in info["tuning"]) > 0
    plan.run()
    torch.cuda.synchronize()
    for b, d in zip(bs, dev):
        got = d[0].cpu().numpy()
        assert np.array_equal(got, _single(cm, torch, b, dms, 64, cm.PREC_OZAKI_INT8))
        assert normwise(got, _single(cm, torch, b, dms, 64)) < 1e-12
    # an SCF step: new D contents, rho zeroed, run again through the same graph
    dms2 = dms + 1e-3 * (dms + dms.transpose(0, 2, 1))
    ddms.copy_(torch.from_numpy(dms2))
    for d in dev:
        d[0].zero_()
    plan.run()
    torch.cuda.synchronize()
    for b, d in zip(bs, dev):
        b2 = dict(b, rho0=np.zeros_like(b["rho0"]))
        assert normwise(d[0].cpu().numpy(), _single(cm, torch, b2, dms2, 64)) < 1e-12
    plan.close()


@pytest.mark.parametrize("form", ["row", "pair"])
@pytest.mark.parametrize("graph", [True, False])
def test_split_plan_of_one_batch(cm, wl, tmp_path, monkeypatch, form, graph):
    """A plan of one batch (the server's plans; the pair form builds it with
    no host round trip: the device's work list, partial offsets from a device
    scan): bit for bit the single split call on two runs with a general D;
    with a symmetric D (the half contraction) within 1e-12 of FP64."""
    import torch
    monkeypatch.setenv("CFGMM_AUTOTUNE_CACHE", str(tmp_path / "tune.txt"))
    monkeypatch.setenv("CFGMM_SPLIT_FORM", form)
    rng = np.random.default_rng(41)
    nao, ngrid, blk, nset = 300, 3000, 64, 2
    nblk = -(-ngrid // blk)
    tab = (rng.random((nao, nblk)) < 0.35).astype(np.uint8)
    phi = rng.standard_normal((nao, ngrid))
    phi[~wl.expand_mask(tab, ngrid, blk)] = 0.0
    dms = rng.uniform(-1, 1, (nset, nao, nao))  # general: no half contraction
    b = dict(lhs=phi, rhs=phi, tab=tab, nset=nset, rho0=rng.standard_normal((nset, ngrid)),
             ngrid=ngrid)
    dev, ddms = _device(torch, [b], dms)
    plan = cm.AodmPlan(dev, ddms, blksize=blk, precision=cm.PREC_OZAKI_INT8, graph=graph)
    plan.run()
    torch.cuda.synchronize()
    want = _single(cm, torch, b, dms, blk, cm.PREC_OZAKI_INT8)
    assert np.array_equal(dev[0][0].cpu().numpy(), want)
    dev[0][0].copy_(torch.from_numpy(b["rho0"]))
    plan.run()
    torch.cuda.synchronize()
    assert np.array_equal(dev[0][0].cpu().numpy(), want)
    assert normwise(want, _single(cm, torch, b, dms, blk)) < 1e-12
    plan.close()
    sdms = wl.sym_dms(rng, nset, nao)  # symmetric: the half contraction
    dev, ddms = _device(torch, [b], sdms)
    plan = cm.AodmPlan(dev, ddms, blksize=blk, precision=cm.PREC_OZAKI_INT8, graph=graph)
    plan.run()
    torch.cuda.synchronize()
    assert normwise(dev[0][0].cpu().numpy(), _single(cm, torch, b, sdms, blk)) < 1e-12
    plan.close()


def test_plan_rejections(cm, wl):
    import torch
    bs, dms = _batches(wl, torch, 4, 2, nset_max=2)
    dev, ddms = _device(torch, bs, dms)
    with pytest.raises(ValueError):
        cm.AodmPlan(dev, ddms, precision=7)
    bad = [(d[0], d[1], d[2], d[3], 3) for d in dev]  # nset above nset_max
    with pytest.raises(ValueError):
        cm.AodmPlan(bad, ddms)


@pytest.mark.parametrize("precision", [0, 1])
def test_plan_symmetric_d_with_two_phi_arrays(cm, wl, precision):
    """Plans over batches whose phi_lhs and phi_rhs differ, with a symmetric D:
    the full contraction runs (the half one needs one phi array per batch), so
    the plan matches the single calls."""
    import torch
    bs, dms = _batches(wl, torch, 5, 9)
    dms = np.ascontiguousarray(0.5 * (dms + dms.transpose(0, 2, 1)))
    dev, ddms = _device(torch, bs, dms)
    plan = cm.AodmPlan(dev, ddms, blksize=64, precision=precision, graph=False, tune=False)
    plan.run()
    torch.cuda.synchronize()
    for b, d in zip(bs, dev):
        assert normwise(d[0].cpu().numpy(), _single(cm, torch, b, dms, 64, precision)) < 1e-12
    plan.close()
