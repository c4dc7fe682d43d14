"""GPU tests of the serving loop (cfgmm_server_*): continuous batching of
density requests from several molecules under an HBM budget.

Every result must equal the single-call contraction within the path's bound
(FP64 1e-13, split 1e-12), and be the same bit for bit whether the request
ran alone or in a mix of concurrent requests from other molecules.
"""
import numpy as np
import pytest

from conftest import normwise

pytestmark = pytest.mark.gpu
WAIT = 120.0


def _molecules(wl, seed, n, blk=64):
    rng = np.random.default_rng(seed)
    mols = []
    for i in range(n):
        nao = int(rng.integers(40, 220))
        ngrid = int(rng.integers(300, 3000))
        nblk = -(-ngrid // blk)
        tab = (rng.random((nao, nblk)) < rng.uniform(0.1, 0.7)).astype(np.uint8)
        ao = rng.standard_normal((nao, ngrid))
        ao[~wl.expand_mask(tab, ngrid, blk)] = 0.0
        nset = int(rng.integers(1, 4))
        d0 = wl.sym_dms(rng, nset, nao)
        steps = [d0]
        for _ in range(2):  # SCF-like steps
            steps.append(steps[-1] + 1e-3 * wl.sym_dms(rng, nset, nao))
        mols.append(dict(ao=ao, tab=tab, nset=nset, dms=steps))
    return mols


def _single(cm, m, dms, blk=64, precision=0):
    nao, ngrid = m["ao"].shape
    rho = np.zeros((m["nset"], ngrid))
    cm.aodmao2rho_ex(rho, dms, m["ao"], m["ao"], (nao, ngrid), (nao, ngrid), m["nset"], m["tab"],
                     m["tab"].shape[1], blk, precision)
    return rho


def _serve(cm, srv, mols, concurrent):
    ids = [srv.open(m["ao"], m["tab"], m["nset"]) for m in mols]
    out = [[np.full((m["nset"], m["ao"].shape[1]), np.nan) for _ in m["dms"]] for m in mols]
    if concurrent:  # interleave every molecule's requests
        tickets = []
        for step in range(3):
            for i, m in enumerate(mols):
                tickets.append(srv.submit(ids[i], m["dms"][step], out[i][step]))
        for t in tickets:
            srv.wait(t, WAIT)
    else:  # one request at a time
        for i, m in enumerate(mols):
            for step in range(3):
                srv.wait(srv.submit(ids[i], m["dms"][step], out[i][step]), WAIT)
    for i in ids:
        srv.close(i)
    return out


@pytest.mark.parametrize("precision,tol", [(0, 1e-13), (1, 1e-12)])
def test_server_alone_and_in_the_mix(cm, wl, tmp_path, monkeypatch, precision, tol):
    monkeypatch.setenv("CFGMM_AUTOTUNE_CACHE", str(tmp_path / "tune.txt"))
    mols = _molecules(wl, 7 + precision, 6)
    srv = cm.Server(8 << 30, nslots=4, precision=precision)
    alone = _serve(cm, srv, mols, concurrent=False)
    mix = _serve(cm, srv, mols, concurrent=True)
    for m, a, b in zip(mols, alone, mix):
        for step in range(3):
            assert np.array_equal(a[step], b[step])  # bit for bit
            assert normwise(a[step], _single(cm, m, m["dms"][step])) < tol
    st = srv.stats()
    assert st["completed"] == 2 * 3 * len(mols) and st["failed"] == 0
    assert st["latency_ms"]["p99"] >= st["latency_ms"]["p50"] > 0
    srv.shutdown()


@pytest.mark.parametrize("precision,tol", [(0, 1e-13), (1, 1e-12)])
def test_server_requests_overlap_on_the_device(cm, wl, tmp_path, monkeypatch, precision, tol):
    """Four molecules of 300-450 AOs on 262144 points each (device-evaluated
    phi, density 0.4): a request's device work (milliseconds) outlasts its
    submission (a copy of its 2 D matrices), so with two requests per
    molecule submitted at once, requests of different molecules are enqueued
    on their slot streams together -- the server's max_inflight stat reaches
    2 or more -- and every result matches the single call."""
    import time
    import torch
    monkeypatch.setenv("CFGMM_AUTOTUNE_CACHE", str(tmp_path / "tune.txt"))
    ngrid = 262144
    mols = []
    for i, nao in enumerate((300, 350, 400, 450)):
        mol = wl.molecule(50 + i, nao=nao, nshell=2 * int(nao / 11.14), natom=nao // 20,
                          box_angstrom=8.0)
        pts = wl.grid_points(np.random.default_rng(60 + i), mol, ngrid, 64)
        ao, tab = wl.device_grid(cm, wl.DeviceMolecule(mol), pts, 64, 0.4)
        dms = [wl.sym_dms(np.random.default_rng(70 + 3 * i + k), 2, nao) for k in range(3)]
        mols.append(dict(ao=ao, tab=tab, dms=dms))
    srv = cm.Server(24 << 30, nslots=4, precision=precision)
    try:
        ids = [srv.open(m["ao"], m["tab"], 2) for m in mols]
        for i, m in zip(ids, mols):  # resident, plans built and tuned
            srv.wait(srv.submit(i, m["dms"][0], np.zeros((2, ngrid))), WAIT)
        outs, tickets = [], []
        for step in (1, 2):
            for i, m in zip(ids, mols):
                o = np.zeros((2, ngrid))
                outs.append((m, step, o))
                tickets.append(srv.submit(i, m["dms"][step], o))
        for t in tickets:
            srv.wait(t, WAIT)
        st = srv.stats()
        for i in ids:
            srv.close(i)
    finally:
        srv.shutdown()
    assert st["failed"] == 0 and st["max_inflight"] >= 2, st
    for m, step, o in outs:
        ref = torch.zeros(2, ngrid, dtype=torch.float64, device="cuda")
        nao = m["ao"].shape[0]
        cm.aodmao2rho_ex(ref, torch.from_numpy(m["dms"][step]).cuda(), m["ao"], m["ao"],
                         (nao, ngrid), (nao, ngrid), 2, m["tab"], m["tab"].shape[1], 64, 0)
        assert normwise(o, ref.cpu().numpy()) < tol


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "split"])
def test_server_device_resident_requests(cm, wl, precision):
    """cfgmm_server_submit_dev: D and rho on the device (an SCF loop kept on
    the GPU).  Each step's D is written on the submitting stream after the
    previous result; the results equal, bit for bit, the host-memory requests
    of the same D matrices on the same server."""
    import torch
    mols = _molecules(wl, 11 + precision, 3)
    srv = cm.Server(8 << 30, nslots=4, precision=precision)
    try:
        ids = [srv.open(m["ao"], m["tab"], m["nset"]) for m in mols]
        host, dev = [], []
        for i, m in zip(ids, mols):
            rh = []
            for step in range(3):
                o = np.zeros((m["nset"], m["ao"].shape[1]))
                srv.wait(srv.submit(i, m["dms"][step], o), WAIT)
                rh.append(o)
            host.append(rh)
        side = torch.cuda.Stream()
        with torch.cuda.stream(side):
            for i, m in zip(ids, mols):
                d = torch.from_numpy(m["dms"][0]).cuda()
                outs = []
                for step in range(3):
                    rho = torch.full((m["nset"], m["ao"].shape[1]), float("nan"),
                                     dtype=torch.float64, device="cuda")
                    srv.wait(srv.submit(i, d, rho), WAIT)
                    outs.append(rho)
                    if step < 2:  # the next step's D, written on the submitting stream
                        d = torch.empty_like(d)
                        d.copy_(torch.from_numpy(m["dms"][step + 1]))
                dev.append(outs)
        torch.cuda.synchronize()
        for i in ids:
            srv.close(i)
        st = srv.stats()
    finally:
        srv.shutdown()
    assert st["failed"] == 0
    for m, rh, rd in zip(mols, host, dev):
        for step in range(3):
            assert np.array_equal(rd[step].cpu().numpy(), rh[step])
    with pytest.raises(ValueError):  # device D with a host rho
        srv2 = cm.Server(1 << 30, nslots=1)
        try:
            i = srv2.open(mols[0]["ao"], mols[0]["tab"], mols[0]["nset"])
            srv2.submit(i, torch.from_numpy(mols[0]["dms"][0]).cuda(),
                        np.zeros((mols[0]["nset"], mols[0]["ao"].shape[1])))
        finally:
            srv2.shutdown()


@pytest.mark.timeout(900)
@pytest.mark.parametrize("form", ["row", "pair"])
def test_server_saturated_device_scf(cm, wl, monkeypatch, form):
    """Every molecule's SCF loop at once with D and rho on the device, each
    client on its own thread and stream (the serving bench's saturated device
    pass), in split precision with the given form forced: every request
    completes, none fails, and each result matches the FP64 single call
    within 1e-12.  The server's completion callback takes no lock; one that
    waited on the server mutex deadlocked this pattern against the worker's
    CUDA calls."""
    import threading
    import torch
    monkeypatch.setenv("CFGMM_SPLIT_FORM", form)
    mols = _molecules(wl, 31, 8)
    srv = cm.Server(8 << 30, nslots=8, precision=1)
    results, errors = [None] * len(mols), []

    def client(k):
        try:
            m = mols[k]
            i = srv.open(m["ao"], m["tab"], m["nset"])
            side = torch.cuda.Stream()
            outs = []
            with torch.cuda.stream(side):
                for step in range(3):
                    d = torch.from_numpy(m["dms"][step]).cuda()
                    rho = torch.full((m["nset"], m["ao"].shape[1]), float("nan"),
                                     dtype=torch.float64, device="cuda")
                    srv.wait(srv.submit(i, d, rho), WAIT)
                    outs.append(rho)
            side.synchronize()
            srv.close(i)
            results[k] = [o.cpu().numpy() for o in outs]
        except Exception as e:  # reported below, on the test's thread
            errors.append(e)

    try:
        th = [threading.Thread(target=client, args=(k,)) for k in range(len(mols))]
        for t in th:
            t.start()
        for t in th:
            t.join()
        st = srv.stats()
    finally:
        srv.shutdown()
    assert not errors, errors
    assert st["failed"] == 0 and st["completed"] == 3 * len(mols), st
    for m, outs in zip(mols, results):
        for step in range(3):
            assert normwise(outs[step], _single(cm, m, m["dms"][step])) < 1e-12


def test_server_budget_admission(cm, wl):
    """A budget that holds about one molecule: every request still completes,
    molecules are admitted one after another, and the server never holds more
    than its budget."""
    mols = _molecules(wl, 3, 4)
    probe = cm.Server(64 << 30, nslots=2)
    costs = []
    for m in mols:  # cost of each molecule = bytes in use when it alone is resident
        i = probe.open(m["ao"], m["tab"], m["nset"])
        out = np.zeros((m["nset"], m["ao"].shape[1]))
        probe.wait(probe.submit(i, m["dms"][0], out), WAIT)
        costs.append(probe.stats()["used_bytes"])
        probe.close(i)
    probe.shutdown()
    budget = int(max(costs) * 1.5)
    srv = cm.Server(budget, nslots=4)
    out = _serve(cm, srv, mols, concurrent=True)
    st = srv.stats()
    assert st["completed"] == 12 and st["failed"] == 0
    assert st["peak_bytes"] <= budget
    for m, o in zip(mols, out):
        for step in range(3):
            assert normwise(o[step], _single(cm, m, m["dms"][step])) < 1e-13
    with pytest.raises(cm.CfgmmError):  # one molecule above the budget
        big = np.zeros((1000, 4096))
        srv.open(big, np.ones((1000, 64), np.uint8), 3)
    srv.shutdown()


def test_server_staging_outlives_servers(cm, wl):
    """The pinned host staging of D and rho is one process-wide pool: a later
    server reuses the buffers of an earlier one, and cfgmm_release_workspace
    frees the idle ones.  Three servers in turn, with the release between the
    second and the third, give the same results bit for bit."""
    mols = _molecules(wl, 41, 3)
    outs = []
    for k in range(3):
        if k == 2:
            assert cm.lib().cfgmm_release_workspace() == 0
        srv = cm.Server(8 << 30, nslots=4)
        try:
            outs.append(_serve(cm, srv, mols, concurrent=True))
            assert srv.stats()["failed"] == 0
        finally:
            srv.shutdown()
    for k in (1, 2):
        for a, b in zip(outs[0], outs[k]):
            for step in range(3):
                assert np.array_equal(a[step], b[step])


def test_server_device_molecule_and_eviction(cm, wl):
    """Caller-owned device phi used in place; LRU eviction under a small
    budget brings a molecule back for its later requests."""
    import torch
    mols = _molecules(wl, 5, 3)
    probe_cost = []
    srv = cm.Server(64 << 30, nslots=2)
    for m in mols:
        d_ao = torch.from_numpy(m["ao"]).cuda()
        d_tab = torch.from_numpy(m["tab"]).cuda()
        m["dev"] = (d_ao, d_tab)
        i = srv.open(d_ao, d_tab, m["nset"])
        out = np.zeros((m["nset"], m["ao"].shape[1]))
        srv.wait(srv.submit(i, m["dms"][0], out), WAIT)
        assert normwise(out, _single(cm, m, m["dms"][0])) < 1e-13
        probe_cost.append(srv.stats()["used_bytes"])
        srv.close(i)
    srv.shutdown()
    srv = cm.Server(int(max(probe_cost) * 1.2), nslots=1)
    ids = [srv.open(m["dev"][0], m["dev"][1], m["nset"]) for m in mols]
    outs = []
    for step in range(3):  # round robin: each step needs the molecule back
        for i, m in zip(ids, mols):
            o = np.zeros((m["nset"], m["ao"].shape[1]))
            srv.wait(srv.submit(i, m["dms"][step], o), WAIT)
            outs.append((m, step, o))
    st = srv.stats()
    assert st["evictions"] >= 2 and st["admitted_molecules"] >= 4
    for m, step, o in outs:
        assert normwise(o, _single(cm, m, m["dms"][step])) < 1e-13
    for i in ids:
        srv.close(i)
    srv.shutdown()


def test_server_shells(cm, wl, oracle):
    """phi evaluated on the device from shells: with every tile kept the
    result matches the oracle on numpy-evaluated phi; with 30 % of the tiles
    repeated requests give the same bits."""
    mol = wl.molecule(2, nao=120, nshell=24, natom=8, box_angstrom=6.0)
    pts = wl.grid_points(np.random.default_rng(2), mol, 1500, 64)
    srv = cm.Server(8 << 30, nslots=2)
    args = (pts, mol.shell_xyz, mol.shell_l, mol.alpha, mol.norm)
    full = srv.open_shells(*args, 1.0, 2)
    part = srv.open_shells(*args, 0.3, 2)
    dms = wl.sym_dms(np.random.default_rng(3), 2, mol.nao)
    r_full = np.zeros((2, len(pts)))
    r_part = [np.zeros((2, len(pts))) for _ in range(2)]
    t = [srv.submit(full, dms, r_full), srv.submit(part, dms, r_part[0]),
         srv.submit(part, dms, r_part[1])]
    for x in t:
        srv.wait(x, WAIT)
    ao = wl.eval_ao_numpy(mol, pts)
    nblk = -(-len(pts) // 64)
    ref = np.zeros((2, len(pts)))
    oracle.aodmao2rho(ref, dms, ao, ao, (mol.nao, len(pts)), (mol.nao, len(pts)), 2,
                      np.ones((mol.nao, nblk), np.uint8), nblk, 64)
    assert normwise(r_full, ref) < 1e-12
    assert np.array_equal(r_part[0], r_part[1]) and np.isfinite(r_part[0]).all()
    assert np.abs(r_part[0]).max() > 0
    srv.close(full)
    srv.close(part)
    srv.shutdown()


def test_server_rejections(cm, wl):
    srv = cm.Server(1 << 30, nslots=1)
    m = _molecules(wl, 1, 1)[0]
    i = srv.open(m["ao"], m["tab"], m["nset"])
    with pytest.raises(ValueError):  # nset above the molecule's nset_max
        srv.submit(i, np.zeros((m["nset"] + 1,) + m["dms"][0].shape[1:]),
                   np.zeros((m["nset"] + 1, m["ao"].shape[1])))
    srv.close(i)
    with pytest.raises(ValueError):  # closed molecule
        srv.submit(i, m["dms"][0], np.zeros((m["nset"], m["ao"].shape[1])))
    with pytest.raises(ValueError):
        srv.wait(12345, 1.0)
    srv.shutdown()
