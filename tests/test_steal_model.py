"""The batched kernel's work-stealing protocol as an interleaving model on the CPU.

Each warp of batched.cu's search kernel is modelled by the lane-0 logic of its stealing code,
one shared-memory operation per model step, and a seeded scheduler interleaves the warps at
random.  The model follows the kernel's operations and their order:

- a busy warp that reads a non-zero hungry count snapshots the ring's head and tail (one
  8-byte word), computes the room `min(32 x hungry, cap / 2) - (tail - head)`, claims slots by a
  compare-and-swap on the tail against its snapshot, then per claimed slot waits for the turn
  word to read 2 x lap, writes the row and releases the slot with turn 2 x lap + 1;
- a warp that runs out of work adds itself to the hungry count and polls: with rows in the ring
  it claims up to 32 by a compare-and-swap on the head, waits per slot for turn 2 x lap + 1,
  reads the row, hands the slot back with 2 x lap + 2, and only then leaves the hungry count;
  with an empty ring it leaves the kernel once the hungry count equals the started count.

Rows are abstract amounts of work; a published row is half of a row the busy warp holds.  The
checks: every unit of work is done exactly once, the ring never holds more than half its slots,
every warp leaves, and the ring is empty at the end -- whatever the interleaving.  The model
also counts the termination window the kernel's design accepts (a warp leaves while a warp that
has just taken rows still holds them): the count stays exact, the rows finish on that warp."""
import random

import pytest


class Model:
    def __init__(self, seed, warps, cap, items, donate_every=3, early_unregister=False):
        self.rng = random.Random(seed)
        self.early_unregister = early_unregister  # the variant that leaves the hungry count first
        self.cap = cap
        self.head = self.tail = 0
        self.turn = [0] * cap
        self.slot = [None] * cap
        self.hungry = 0
        self.started = warps
        self.donate_every = donate_every
        self.done_units = 0
        self.done_by = [0] * warps
        self.max_fill = 0
        self.window_exits = 0
        self.warps = [self._warp(w, items[w::warps]) for w in range(warps)]
        self.holding = [False] * warps  # took ring rows, still counted hungry

    def _ring(self):
        return self.head, self.tail

    def _warp(self, w, rows):
        """Generator: yields after each shared-memory operation."""
        rows = [r for r in rows if r > 0]
        rounds = 0
        while True:
            # busy: work on the rows, publishing now and then
            while rows:
                rows[-1] -= 1
                self.done_units += 1
                self.done_by[w] += 1
                if rows[-1] == 0:
                    rows.pop()
                yield
                rounds += 1
                if rounds % self.donate_every or not rows:
                    continue
                g = self.hungry
                yield
                if not g:
                    continue
                h, t = self._ring()
                yield
                need = min(32 * g, self.cap // 2)
                spare = [i for i, r in enumerate(rows) if r >= 2]
                if t - h >= need or not spare:
                    continue
                k = min(len(spare), need - (t - h))
                if self.tail != t:  # compare-and-swap lost: look again next time
                    yield
                    continue
                self.tail = t + k
                self.max_fill = max(self.max_fill, self.tail - self.head)
                yield
                for j in range(k):
                    idx = t + j
                    lap = idx // self.cap
                    while self.turn[idx % self.cap] != 2 * lap:  # the slot's previous lap is read
                        yield
                    i = spare[j]
                    give = rows[i] // 2
                    rows[i] -= give
                    self.slot[idx % self.cap] = give
                    self.turn[idx % self.cap] = 2 * lap + 1
                    yield
            # hungry
            self.hungry += 1
            yield
            while True:
                h, t = self._ring()
                yield
                if t != h:
                    want = min(t - h, 32)
                    if self.early_unregister:  # leave the hungry count before the take
                        self.hungry -= 1
                        yield
                    if self.head != h:  # another warp took rows first
                        if self.early_unregister:
                            self.hungry += 1
                        yield
                        continue
                    self.head = h + want
                    self.holding[w] = True  # rows taken, not yet being searched
                    yield
                    for j in range(want):
                        idx = h + j
                        lap = idx // self.cap
                        while self.turn[idx % self.cap] != 2 * lap + 1:
                            yield
                        rows.append(self.slot[idx % self.cap])
                        self.slot[idx % self.cap] = None
                        self.turn[idx % self.cap] = 2 * lap + 2
                        yield
                    if not self.early_unregister:
                        self.hungry -= 1
                    self.holding[w] = False
                    yield
                    break
                g = self.hungry
                yield
                if g == self.started:
                    if any(self.holding):
                        self.window_exits += 1
                    return
                yield

    def run(self, max_steps=2_000_000):
        live = list(range(len(self.warps)))
        for _ in range(max_steps):
            if not live:
                return
            w = self.rng.choice(live)
            try:
                next(self.warps[w])
            except StopIteration:
                live.remove(w)
        raise AssertionError("the model did not terminate")


@pytest.mark.parametrize("early_unregister", [False, True])
@pytest.mark.parametrize("seed", range(60))
def test_steal_protocol_is_exact_under_any_interleaving(seed, early_unregister):
    rng = random.Random(1000 + seed)
    warps = rng.choice([2, 3, 4, 6, 8])
    cap = rng.choice([2, 4, 8, 64])
    # uneven items: most warps get little, a few get long subtrees
    items = [rng.choice([0, 1, 3, 10, 200, 1500]) for _ in range(warps * rng.choice([1, 2, 3]))]
    m = Model(seed, warps, cap, items, donate_every=rng.choice([1, 3, 16]), early_unregister=early_unregister)
    m.run()
    assert m.done_units == sum(items)       # every unit once: no row lost or duplicated
    assert m.head == m.tail                 # the ring is empty at the end
    assert all(s is None for s in m.slot)
    assert m.max_fill <= cap // 2           # producers never fill more than half the ring
    assert m.hungry == m.started            # every warp ended hungry and left


def test_steal_protocol_spreads_a_long_subtree():
    # one long item on one warp: the other warps live off the ring and do most of the work
    m = Model(7, 8, 64, [20000] + [0] * 7, donate_every=2)
    m.run()
    assert m.done_units == 20000 and m.head == m.tail
    assert m.done_by[0] < 0.5 * 20000 and sum(1 for x in m.done_by if x > 0) == 8


def test_termination_window_keeps_the_count():
    # in some interleavings warps leave while another still holds rows it has just taken (the
    # window the kernel accepts: 7 such exits in 2 of these 40 runs); the count stays exact in
    # every run
    windows = 0
    for seed in range(40):
        m = Model(seed, 6, 8, [400, 5, 5, 900, 0, 50], donate_every=1)
        m.run()
        assert m.done_units == 1360 and m.head == m.tail
        windows += m.window_exits
    assert windows > 0


def test_leaving_the_hungry_count_before_the_take_closes_the_window():
    # the variant (not built in the kernel): a poller leaves the hungry count before its
    # compare-and-swap on the head and joins it again if that fails; no warp then leaves while
    # another holds taken rows, and the count stays exact
    for seed in range(40):
        m = Model(seed, 6, 8, [400, 5, 5, 900, 0, 50], donate_every=1, early_unregister=True)
        m.run()
        assert m.done_units == 1360 and m.head == m.tail and m.hungry == m.started
        assert m.window_exits == 0
