"""The fused kernel's synchronisation protocol, modelled on the CPU.

fused_tc.cu runs 16 producer warps, a TMA thread and an MMA thread over a
ring of NST stages with mbarriers whose waits test a phase's parity only.
This test replays that protocol as a discrete-event model with random and
adversarial schedules and checks, for every schedule:

* it ends (no deadlock);
* every parity wait that passes does so because the intended phase has
  completed (a waiter two phases behind or ahead would pass or block
  wrongly);
* every completed phase of a k-step barrier holds the arrivals of one K
  block only;
* no data hazard: a chunk is written into a stage only after the MMAs of
  the block that used it last are done; a producer reads its block's
  record; an MMA reads a complete A tile and its own block's coefficient
  tile; a coefficient tile or record is reloaded only once its previous
  block no longer needs it.

Forms: three accumulators (two stages, a coefficient tile per stage) and
wide MO tiles (a single coefficient tile, two or three stages).  Schedules:
random, adversarial (each actor moves with probability 0.15 a step), and
with one producer warp held back until nothing else can move.  Two variants
known to be wrong must be caught: chunks of skipped k-steps arriving
themselves without waiting for the record, while each record is loaded as
soon as every chunk of the block two back has arrived (a skipped chunk of a
later block can then arrive before the TMA thread's parity wait for the
earlier phase, which falls two phases behind); and chunks of skipped
k-steps waiting on the stage barrier's parity alone (the block's MMAs need
none of their arrivals, so a warp held back can reach its wait after the
phase it waits for and the next have completed, and waits for the stage's
next use; the kernel's wait also ends on the count of released blocks that
the TMA thread publishes).
"""
import random

import pytest

CHUNKS, KSTEPS, WARPS = 16, 4, 16
PER_K = CHUNKS // KSTEPS


class ProtocolViolation(AssertionError):
    pass


class Bar:
    def __init__(self, name, count):
        self.name, self.count, self.pending, self.phase, self.tx = name, count, count, 0, 0
        self.tags = []

    def arrive(self, n=1, tag=None):
        if tag is not None:
            self.tags.append(tag)
        self.pending -= n
        if self.pending < 0:
            raise ProtocolViolation(f"{self.name}: too many arrivals in phase {self.phase}")
        self._complete()

    def expect(self, nbytes):
        self.tx += nbytes

    def land(self, nbytes):
        self.tx -= nbytes
        self._complete()

    def _complete(self):
        if self.pending == 0 and self.tx == 0:
            if len(set(self.tags)) > 1:
                raise ProtocolViolation(f"{self.name}: phase {self.phase} mixes blocks {self.tags}")
            self.phase += 1
            self.pending, self.tags = self.count, []

    def wait(self, k, late_ok=False):
        """A parity wait for phase k (k < 0: the phase before the first).
        late_ok: the caller also ends its wait by other means (a counter),
        so a parity wait that reads the barrier a phase late is no fault."""
        passed = (self.phase & 1) != (k & 1)
        if passed and self.phase <= k:
            raise ProtocolViolation(f"{self.name}: wait for phase {k} passed in phase {self.phase}")
        if not passed and self.phase > k and not late_ok:
            raise ProtocolViolation(f"{self.name}: wait for completed phase {k} blocked in phase {self.phase}")
        return passed


def run(masks, seed, nst=2, wide=False, adversarial=False, bad_variant=False, warps=WARPS, dead_parity=False,
        late=None):
    rng = random.Random(seed)
    n = len(masks)
    full = [[Bar(f"full[{s}][{k}]", PER_K) for k in range(KSTEPS)] for s in range(nst)]
    bfull = [Bar(f"bfull[{s}]", 1) for s in range(nst)]
    empty = [Bar(f"empty[{s}]", 1) for s in range(nst)]
    rec = [Bar(f"rec[{s}]", 1) for s in range(nst)]
    a_tile = [dict() for _ in range(nst)]          # stage -> {chunk: block}
    b_tile = {}                                    # coefficient buffer -> block
    rec_slot = [None] * nst
    mma_done, produced = set(), {}
    pending, claim = [], [warps]
    clock = [0]
    released = [0]   # blocks whose MMAs the TMA thread has seen done (a counter in shared memory)

    def live(it, c):
        m = masks[it] or 0xF
        return (m >> (c // PER_K)) & 1

    def copy(bar, apply):
        bar.expect(1)
        bar.arrive()
        pending.append((clock[0] + rng.randint(1, 30), lambda: (apply(), bar.land(1))))

    def load_record(it):
        s = it % nst
        def apply():
            old = rec_slot[s]
            if old is not None and any(live(old, c) and (old, c) not in produced for c in range(CHUNKS)):
                raise ProtocolViolation(f"record of block {old} overwritten before its chunks were produced")
            rec_slot[s] = it
        copy(rec[s], apply)

    def load_coef(it):
        key = "B" if wide else it % nst
        def apply():
            old = b_tile.get(key)
            if old is not None and old not in mma_done:
                raise ProtocolViolation(f"coefficients of block {old} overwritten before its MMAs were done")
            b_tile[key] = it
        copy(bfull[it % nst], apply)

    def producer(w):
        q = w
        while q < n * CHUNKS:
            it, c = divmod(q, CHUNKS)
            s, k = it % nst, it // nst
            if live(it, c) or dead_parity or bad_variant:
                yield lambda: empty[s].wait(k - 1)
            else:   # a chunk of a skipped k-step: the stage barrier, or the count of released blocks
                yield lambda: empty[s].wait(k - 1, late_ok=True) or released[0] >= it - nst + 1
            if live(it, c):
                yield lambda: rec[s].wait(k)
                if it >= nst and (it - nst) not in mma_done:
                    raise ProtocolViolation(f"chunk of block {it} written while block {it - nst} is read")
                if rec_slot[s] != it:
                    raise ProtocolViolation(f"block {it} produced from the record of block {rec_slot[s]}")
                for _ in range(rng.randint(1, 12)):
                    yield lambda: True
                a_tile[s][c] = it
                produced[(it, c)] = True
                full[s][c // PER_K].arrive(tag=it)
            elif bad_variant:
                full[s][c // PER_K].arrive(tag=it)
            q = claim[0]
            claim[0] += 1

    def tma():
        pre = min(n, nst)
        for it in range(pre):
            load_record(it)
            if not wide or it == 0:
                load_coef(it)
        if not wide:
            for it in range(pre, n):
                s, k = it % nst, it // nst
                if bad_variant:
                    for kk in range(KSTEPS):
                        yield lambda kk=kk: full[s][kk].wait(k - 1)
                    load_record(it)
                yield lambda: empty[s].wait(k - 1)
                released[0] = it - nst + 1
                if not bad_variant:
                    load_record(it)
                load_coef(it)
        else:
            for it in range(1, n):
                b = it - 1
                yield lambda: empty[b % nst].wait(b // nst)
                released[0] = it
                load_coef(it)
                r = it + nst - 1
                if pre <= r < n:
                    load_record(r)

    def mma():
        for it in range(n):
            s, k = it % nst, it // nst
            yield lambda: bfull[s].wait(k)
            if b_tile.get("B" if wide else s) != it:
                raise ProtocolViolation(f"MMAs of block {it} with the coefficients of another block")
            for kk in range(KSTEPS):
                dead = not live(it, kk * PER_K)
                if dead and not bad_variant:   # the MMA thread arrives for a skipped k-step
                    full[s][kk].arrive(PER_K, tag=it)
                yield lambda kk=kk: full[s][kk].wait(k)
                if not dead and any(a_tile[s].get(c) != it for c in range(kk * PER_K, kk * PER_K + PER_K)):
                    raise ProtocolViolation(f"MMAs of block {it} on an incomplete A tile")
            def done(it=it, s=s):
                mma_done.add(it)
                empty[s].arrive()
            pending.append((clock[0] + rng.randint(1, 10), done))

    actors = [producer(w) for w in range(warps)] + [tma(), mma()]
    cur = [next(a, None) for a in actors]
    while True:
        clock[0] += 1
        due = [p for p in pending if p[0] <= clock[0]]
        pending[:] = [p for p in pending if p[0] > clock[0]]
        for _, f in due:
            f()
        moved = False
        order = [i for i in range(len(actors)) if i != late]
        rng.shuffle(order)
        for i in order:
            if adversarial and rng.random() > 0.15:
                continue
            while cur[i] is not None and cur[i]():
                cur[i] = next(actors[i], None)
                moved = True
                if rng.random() < 0.5:
                    break
        if late is not None and not moved and not pending:   # the late warp runs only when all else waits
            while cur[late] is not None and cur[late]():
                cur[late] = next(actors[late], None)
                moved = True
        if all(c is None for c in cur) and not pending:
            return
        if not moved and not pending and not any(c is not None and c() for c in cur):
            raise ProtocolViolation("deadlock")


def _masks(rng):
    return [rng.choice([0xF, 0x1, 0x8, 0x6, 0x9, 0x3, 0xC, 0x2, 0x4, 0x5, 0xA, 0x7, 0xE]) for _ in range(rng.randint(1, 10))]


@pytest.mark.parametrize("nst,wide", [(2, False), (2, True), (3, True)])
@pytest.mark.parametrize("adversarial", [False, True])
def test_protocol_holds(nst, wide, adversarial):
    for seed in range(150):
        run(_masks(random.Random(seed)), seed, nst=nst, wide=wide, adversarial=adversarial)


@pytest.mark.parametrize("nst,wide", [(2, False), (2, True), (3, True)])
@pytest.mark.parametrize("late", [0, 3, 9])
def test_protocol_holds_with_a_warp_held_back(nst, wide, late):
    for seed in range(40):
        run(_masks(random.Random(seed)), seed, nst=nst, wide=wide, adversarial=seed % 2 == 0, late=late)


def test_known_bad_variant_is_caught():
    failures = 0
    for seed in range(150):
        try:
            run(_masks(random.Random(seed)), seed, nst=2, bad_variant=True)
        except ProtocolViolation:
            failures += 1
    assert failures > 0


def test_parity_only_wait_of_skipped_chunks_is_caught():
    failures = 0
    for seed in range(40):
        try:
            run(_masks(random.Random(seed)), seed, nst=3, wide=True, dead_parity=True, late=0)
        except ProtocolViolation as e:
            assert "blocked" in str(e)
            failures += 1
    assert failures > 0
