"""Synchronisation protocol of oz_mma_kernel (fastmbcui_b200/csrc/matvec_oz.cuh),
model-checked on the CPU.

The kernel's three roles are replayed as coroutines over a model of PTX
mbarriers: a barrier counts completed phases; a phase completes once its
expected arrivals and transaction bytes are in; try_wait.parity(p) succeeds
iff the current phase's parity differs from p.  Bulk copies land, and
tcgen05.commit arrivals fire (in issue order), at random later times.  Random
interleavings of the roles are run for several k-step and chunk counts,
asserting
  * every parity wait answers the question the kernel means to ask (the
    phase it intends has completed: no aliasing two phases ahead);
  * the loader refills an A or B slot only after the MMAs that read its
    previous contents completed;
  * the MMA warp reads a slot only after its copy landed;
  * the first (zero-initialising) MMA of a chunk starts only after the
    accumulator warps folded the previous chunk, and a fold reads a chunk
    only after all its MMAs completed;
  * every role finishes (no deadlock).
The constants are the kernel's: 6 single-plane A slots, 2 B slots, 5 planes
per k-step, 16 k-steps per chunk, 8 accumulator-warp arrivals.
"""
import random

import pytest

A_SLOTS, B_SLOTS, DIGITS, CHUNK_STEPS, ACC_WARPS = 6, 2, 5, 16, 8


class Barrier:
    def __init__(self, name, count):
        self.name, self.count = name, count
        self.completed = 0      # phases completed
        self.pending = count    # arrivals still expected in the current phase
        self.tx = 0             # transaction bytes still expected

    def arrive(self, expect_tx=0):
        self.pending -= 1
        self.tx += expect_tx
        self._maybe_complete()

    def complete_tx(self, b):
        self.tx -= b
        self._maybe_complete()

    def _maybe_complete(self):
        assert self.pending >= 0
        if self.pending == 0 and self.tx == 0:
            self.completed += 1
            self.pending = self.count

    def try_wait(self, parity):
        return (self.completed % 2) != parity


class Model:
    def __init__(self, nks, seed):
        self.rng = random.Random(seed)
        self.nks = nks
        self.nchunks = (nks + CHUNK_STEPS - 1) // CHUNK_STEPS
        self.afull = [Barrier(f"afull{s}", 1) for s in range(A_SLOTS)]
        self.aempty = [Barrier(f"aempty{s}", 1) for s in range(A_SLOTS)]
        self.bfull = [Barrier(f"bfull{s}", 1) for s in range(B_SLOTS)]
        self.bempty = [Barrier(f"bempty{s}", 1) for s in range(B_SLOTS)]
        self.chunk_full = Barrier("chunk_full", 1)
        self.chunk_free = Barrier("chunk_free", ACC_WARPS)
        self.mma_done = Barrier("mma_done", 1)
        self.events = []          # async completions: (kind, payload)
        self.commits = []         # tcgen05.commit queue, fires in order
        # bookkeeping for the invariants
        self.a_content = [None] * A_SLOTS   # use t whose copy is (being) written
        self.a_landed = [False] * A_SLOTS
        self.a_readers_done = [True] * A_SLOTS
        self.b_content = [None] * B_SLOTS
        self.b_landed = [False] * B_SLOTS
        self.b_readers_done = [True] * B_SLOTS
        self.mma_outstanding = 0
        self.chunk_mmas_done = set()
        self.folded = set()

    # --- waits ---------------------------------------------------------
    def wait(self, bar, parity, intended_phase):
        """Kernel-side bounded wait: yields until try_wait succeeds; checks
        that the parity answer equals 'phase intended_phase has completed'."""
        while True:
            ok = bar.try_wait(parity)
            truth = bar.completed > intended_phase if intended_phase >= 0 else True
            assert ok == truth, f"{bar.name}: parity {parity} answers {ok}, phase {intended_phase} done {truth}"
            if ok:
                return
            yield

    # --- roles ---------------------------------------------------------
    def loader(self):
        for ks in range(self.nks):
            sb = ks % B_SLOTS
            yield from self.wait(self.bempty[sb], ((ks // B_SLOTS) & 1) ^ 1, ks // B_SLOTS - 1)
            assert self.b_readers_done[sb], "B slot refilled while its MMAs run"
            self.b_content[sb], self.b_landed[sb] = ks, False
            self.bfull[sb].arrive(expect_tx=1)
            self.events.append(("bcopy", sb))
            yield
            for p in range(DIGITS):
                t = ks * DIGITS + p
                sa = t % A_SLOTS
                yield from self.wait(self.aempty[sa], ((t // A_SLOTS) & 1) ^ 1, t // A_SLOTS - 1)
                assert self.a_readers_done[sa], "A slot refilled while its MMAs run"
                self.a_content[sa], self.a_landed[sa] = t, False
                self.afull[sa].arrive(expect_tx=1)
                self.events.append(("acopy", sa))
                yield
        # drain: the last copies of each ring
        for ks in range(max(0, self.nks - B_SLOTS), self.nks):
            yield from self.wait(self.bfull[ks % B_SLOTS], (ks // B_SLOTS) & 1, ks // B_SLOTS)
        last = self.nks * DIGITS
        for t in range(max(0, last - A_SLOTS), last):
            yield from self.wait(self.afull[t % A_SLOTS], (t // A_SLOTS) & 1, t // A_SLOTS)

    def mma(self):
        for ks in range(self.nks):
            kc, sb = ks % CHUNK_STEPS, ks % B_SLOTS
            yield from self.wait(self.bfull[sb], (ks // B_SLOTS) & 1, ks // B_SLOTS)
            if kc == 0 and ks > 0:
                c = ks // CHUNK_STEPS
                yield from self.wait(self.chunk_free, (c - 1) & 1, c - 1)
                assert (c - 1) in self.folded, "chunk overwritten before its fold"
            assert self.b_landed[sb] and self.b_content[sb] == ks, "B read before it landed"
            self.b_readers_done[sb] = False
            for p in range(DIGITS):
                t = ks * DIGITS + p
                sa = t % A_SLOTS
                yield from self.wait(self.afull[sa], (t // A_SLOTS) & 1, t // A_SLOTS)
                assert self.a_landed[sa] and self.a_content[sa] == t, "A read before it landed"
                self.a_readers_done[sa] = False
                self.mma_outstanding += 1
                self.commits.append(("a", sa))
                yield
            self.commits.append(("b", sb))
            if kc == CHUNK_STEPS - 1 or ks == self.nks - 1:
                self.commits.append(("chunk", ks // CHUNK_STEPS))
            yield
        self.commits.append(("done", None))
        yield from self.wait(self.mma_done, 0, 0)

    def acc(self):
        for c in range(self.nchunks):
            yield from self.wait(self.chunk_full, c & 1, c)
            assert c in self.chunk_mmas_done, "fold before the chunk's MMAs completed"
            self.folded.add(c)
            yield
            if c < self.nchunks - 1:
                for _ in range(ACC_WARPS):
                    self.chunk_free.arrive()
                    yield

    # --- asynchronous completions ----------------------------------------
    def fire_one(self):
        choices = []
        if self.events:
            choices.append("copy")
        if self.commits:
            choices.append("commit")
        if not choices:
            return False
        if self.rng.choice(choices) == "copy":
            kind, s = self.events.pop(self.rng.randrange(len(self.events)))
            if kind == "acopy":
                self.a_landed[s] = True
                self.afull[s].complete_tx(1)
            else:
                self.b_landed[s] = True
                self.bfull[s].complete_tx(1)
        else:
            kind, s = self.commits.pop(0)  # commits fire in issue order
            if kind == "a":
                self.a_readers_done[s] = True
                self.aempty[s].arrive()
            elif kind == "b":
                self.b_readers_done[s] = True
                self.bempty[s].arrive()
            elif kind == "chunk":
                self.chunk_mmas_done.add(s)
                self.chunk_full.arrive()
            else:
                self.mma_done.arrive()
        return True

    def run(self, max_steps=2_000_000):
        roles = {"loader": self.loader(), "mma": self.mma(), "acc": self.acc()}
        for _ in range(max_steps):
            if not roles and not self.events and not self.commits:
                return
            r = self.rng.random()
            if roles and (r < 0.7 or not (self.events or self.commits)):
                name = self.rng.choice(sorted(roles))
                try:
                    next(roles[name])
                except StopIteration:
                    del roles[name]
            else:
                self.fire_one()
        raise AssertionError(f"no progress: roles left {sorted(roles)}")


@pytest.mark.parametrize("nks", [1, 2, 5, 15, 16, 17, 33, 48])
def test_protocol_random_schedules(nks):
    for seed in range(40):
        m = Model(nks, seed)
        m.run()
        assert m.folded == set(range(m.nchunks))
        assert m.mma_done.completed == 1
