"""A host-side model of the barrier protocol of the split AO-DM-AO pair kernel
(`pair_main` in csrc/aodmao2rho_split_pair.cu), run under random
interleavings of its warps.

Actors: the 12 gather/epilogue warps (3 groups of 4), the MMA thread, the
loader thread, the tensor-core engine (executes issued MMAs and commits in
order, at random times) and the bulk-copy engine (lands phi tiles at random
times).  Barriers follow mbarrier semantics: `wait(bar, P)` passes iff the
number of completed phases has parity different from P -- so a wait two
phases early passes falsely, which the model must never need.

Checked on every interleaving: no deadlock; a stage is refilled only after the
MMAs of its previous chunk executed; the MMAs of a chunk read the D digits of
all four warps of the chunk's group and the phi tile of the same chunk; an
item's first MMA runs only after every warp has read the previous item's
accumulators; every group writes its partial sums of every item once.
"""
import random

import pytest

NG, GW = 3, 12
STAGES = 3
RING = 4
AHEAD = 2


class Bar:
    def __init__(self, count):
        self.count, self.pending, self.phase = count, count, 0

    def arrive(self):
        self.pending -= 1
        assert self.pending >= 0
        if self.pending == 0:
            self.phase += 1
            self.pending = self.count

    def passed(self, parity):
        return (self.phase & 1) != parity


class Model:
    def __init__(self, items, rng):
        self.items, self.rng = items, rng  # items: list of (kc0, kc)
        self.full_phi = [Bar(1) for _ in range(STAGES)]
        self.full_d = [Bar(4) for _ in range(STAGES)]
        self.empty = [Bar(1) for _ in range(STAGES)]
        self.acc_full, self.acc_empty, self.drain = Bar(1), Bar(GW), Bar(1)
        self.ifull = [Bar(1) for _ in range(RING)]
        self.iempty = [Bar(GW + 2) for _ in range(RING)]
        self.ring = [None] * RING
        self.stage_d = [dict() for _ in range(STAGES)]  # warp -> seq written
        self.stage_phi = [None] * STAGES
        self.executed = -1          # highest chunk whose MMAs executed
        self.engine = []            # issued MMA work and commits, in order
        self.copies = []            # bulk copies in flight: (stage, seq)
        self.tmem_read = {}         # item -> warps that read its accumulators
        self.tmem_item = None       # item whose MMAs the accumulators hold
        self.sums = []

    # ---- roles (generators yield a predicate to wait on) ----
    def item_of(self, n):
        yield lambda: self.ifull[n % RING].passed((n // RING) & 1)
        t = self.ring[n % RING]
        self.iempty[n % RING].arrive()
        return t

    def gather_warp(self, w):
        grp = w // 4
        state = {"done": -1}

        def stage_free(seq):
            need = seq - STAGES
            while state["done"] < need:
                y = min(state["done"] + STAGES, need)
                yield lambda y=y: self.empty[y % STAGES].passed((y // STAGES) & 1)
                state["done"] = y

        def gather(seq):
            yield from stage_free(seq)
            stg = seq % STAGES
            assert self.executed >= seq - STAGES, "stage refilled before its MMAs ran"
            self.stage_d[stg][w] = seq
            self.full_d[stg].arrive()

        seq0, ahead, nitem = 0, False, 0
        t = yield from self.item_of(0)
        while t is not None:
            kc0, kc = self.items[t]
            c = kc0 + grp + (NG if ahead else 0)
            while c < kc:
                yield from gather(seq0 + c - kc0)
                c += NG
            seq1 = seq0 + kc - kc0
            # the next item's first chunk of the group: loaded before the
            # accumulator wait, stored once the accumulators are read
            tn = yield from self.item_of(nitem + 1)
            ahead = tn is not None and self.items[tn][0] + grp < self.items[tn][1]
            yield lambda n=nitem: self.acc_full.passed(n & 1)
            state["done"] = max(state["done"], seq1 - 1)
            assert self.tmem_item == nitem and self.executed >= seq1 - 1
            self.tmem_read.setdefault(nitem, set()).add(w)
            self.acc_empty.arrive()
            if ahead:
                yield from gather(seq1 + grp)
            if w % 4 == 0:  # the group's partial sums of the item go out
                self.sums.append((nitem, grp))
            seq0, t, nitem = seq1, tn, nitem + 1

    def mma_thread(self):
        seq, nitem = 0, 0
        while True:
            t = yield from self.item_of(nitem)
            if t is None:
                break
            kc0, kc = self.items[t]
            if nitem > 0:
                yield lambda n=nitem: self.acc_empty.passed((n - 1) & 1)
            for c in range(kc0, kc):
                stg, par = seq % STAGES, (seq // STAGES) & 1
                yield lambda s=stg, p=par: self.full_phi[s].passed(p)
                yield lambda s=stg, p=par: self.full_d[s].passed(p)
                grp = (c - kc0) % NG
                want = {w: seq for w in range(4 * grp, 4 * grp + 4)}
                got = {w: self.stage_d[stg].get(w) for w in want}
                assert got == want, f"chunk {seq}: D digits {got}"
                assert self.stage_phi[stg] == seq, "phi tile of another chunk"
                self.engine.append(("mma", seq, nitem, c == kc0))
                self.engine.append(("commit", self.empty[stg]))
                seq += 1
            self.engine.append(("commit", self.acc_full))
            nitem += 1
        self.engine.append(("commit", self.drain))
        yield lambda: self.drain.passed(0)

    def loader_thread(self):
        seq, drawn, ended = 0, 0, False
        tq = [None] * RING
        issued = [0] * STAGES
        n = 0
        while True:
            while not ended and drawn <= n + AHEAD:  # items drawn AHEAD ahead
                slot = drawn % RING
                if drawn >= RING:
                    yield lambda s=slot, d=drawn: self.iempty[s].passed(((d // RING) - 1) & 1)
                t = drawn if drawn < len(self.items) else None
                self.ring[slot] = tq[slot] = t
                self.ifull[slot].arrive()
                self.iempty[slot].arrive()
                ended = t is None
                drawn += 1
            t = tq[n % RING]
            if t is None:
                break
            kc0, kc = self.items[t]
            for c in range(kc0, kc):
                stg, use = seq % STAGES, seq // STAGES
                if use > 0:
                    yield lambda s=stg, u=use: self.empty[s].passed((u - 1) & 1)
                assert self.executed >= seq - STAGES
                self.copies.append((stg, seq))
                issued[stg] += 1
                seq += 1
            n += 1
        for s in range(STAGES):
            if issued[s]:
                yield lambda s=s: self.full_phi[s].passed((issued[s] - 1) & 1)

    def tensor_engine(self):
        while True:
            yield lambda: bool(self.engine) or self.done_issuing
            if not self.engine:
                return
            op = self.engine.pop(0)
            if op[0] == "mma":
                _, seq, nitem, first = op
                if first:  # overwrites the accumulators: the last item is read
                    if nitem > 0:
                        assert self.tmem_read.get(nitem - 1) == set(range(GW)), "TMEM overwritten"
                    self.tmem_item = nitem
                assert seq == self.executed + 1
                self.executed = seq
            else:
                op[1].arrive()

    def copy_engine(self):
        while True:
            yield lambda: bool(self.copies) or self.done_loading
            if not self.copies:
                return
            stg, seq = self.copies.pop(self.rng.randrange(len(self.copies)))
            self.stage_phi[stg] = seq
            self.full_phi[stg].arrive()

    def run(self):
        self.done_issuing = self.done_loading = False
        actors = {f"g{w}": self.gather_warp(w) for w in range(GW)}
        actors["mma"], actors["load"] = self.mma_thread(), self.loader_thread()
        engines = {"tc": self.tensor_engine(), "copy": self.copy_engine()}
        waits = {}
        for name, gen in list(actors.items()) + list(engines.items()):
            waits[name] = next(gen)
        live = dict(actors, **engines)
        while live:
            self.done_issuing = "mma" not in live
            self.done_loading = "load" not in live
            ready = [k for k in live if waits[k]()]
            assert ready, f"deadlock: waiting {sorted(live)}"
            k = self.rng.choice(ready)
            try:
                waits[k] = live[k].send(None)
            except StopIteration:
                del live[k]
        assert sorted(self.sums) == [(n, g) for n in range(len(self.items)) for g in range(NG)]


def _items(rng, n):
    out = []
    for _ in range(n):
        kc0 = rng.randrange(0, 6)
        out.append((kc0, kc0 + rng.choice([1, 1, 2, 3, 4, 5, 7, 9])))
    return out


@pytest.mark.parametrize("seed", range(60))
def test_pair_protocol_random_interleavings(seed):
    rng = random.Random(seed)
    Model(_items(rng, rng.randrange(1, 14)), rng).run()


def test_a_wait_two_phases_early_passes_falsely():
    """The model's barriers alias phases by parity like mbarriers do, so the
    in-order stepping of the stage waits is what keeps them exact."""
    b = Bar(1)
    assert not b.passed(0)
    b.arrive()
    b.arrive()  # two phases completed
    assert b.passed(1)  # phase 1 done: correct
    assert not b.passed(0)  # phase 2 (parity 0) not done: correct
    b2 = Bar(1)
    assert b2.passed(1)  # "phase 1" before any phase completed: aliasing
