"""A CPU model of the search step's machine (the shared-memory stack of pending rows, entry
counting and the dead-end filter of search_step.cuh), written out in Python and checked
against the oracle's counts and nodes on whole pools.  It pins the arithmetic the step's PTX
implements -- which candidates the filter may drop without a step -- and the share of
placements it removes from the step loop, independently of a GPU."""
import numpy as np
import pytest


def drop_leaves(a, nc, l, r):
    g = nc & ~(((l << 1) & 0xFFFFFFFF) | (r >> 1))
    if (g & -g) != g:
        return a
    return a & ~((g * 7) >> 1) if g else 0


def run_machine(state, filtered=True):
    """(count, nodes, steps, pushes) of one state's search."""
    n = int(state["n"])
    nc = ((1 << n) - 1) & ~int(state["cols"])
    l, r = int(state["ldiag"]), int(state["rdiag"])
    stack = []
    count = nodes = steps = pushes = 0

    def enter(nc, l, r):
        nonlocal count, nodes
        a = nc & ~(l | r)
        pc = bin(a).count("1")
        nodes += pc
        if (nc & (nc - 1)) == 0:
            count += pc + (nc == 0)
        return drop_leaves(a, nc, l, r) if filtered else a

    a = enter(nc, l, r)
    while True:
        if a == 0:
            if not stack:
                break
            a, nc, l, r = stack.pop()
        b = a & -a
        a -= b
        if a:
            stack.append((a, nc, l, r))
            pushes += 1
        nc, l, r = nc - b, ((l + b) << 1) & 0xFFFFFFFF, (r + b) >> 1
        steps += 1
        a = enter(nc, l, r)
    return count, nodes, steps, pushes


@pytest.mark.parametrize("n,d", [(8, 2), (10, 3), (11, 4), (12, 3)])
def test_filtered_machine_matches_oracle(nqb, nqo, n, d):
    pool = nqb.generate_pool(n, d)
    want, want_nodes = nqo.solve_states(pool)
    got = [run_machine(s) for s in pool]
    assert [g[0] * int(s["weight"]) for g, s in zip(got, pool)] == list(want)
    assert sum(g[1] for g in got) == want_nodes


def test_filter_removes_a_third_of_the_steps(nqb):
    pool = nqb.generate_pool(12, 3)
    plain = [run_machine(s, filtered=False) for s in pool]
    filt = [run_machine(s) for s in pool]
    nodes = sum(p[1] for p in plain)
    assert nodes == sum(f[1] for f in filt)
    assert sum(p[2] for p in plain) == nodes  # unfiltered: one step per placement
    share = sum(f[2] for f in filt) / nodes
    assert 0.60 < share < 0.72, share      # ~0.66 at N=12..21
    assert sum(f[3] for f in filt) < 0.75 * sum(p[3] for p in plain)


def test_dropped_candidates_are_dead_ends():
    # exhaustive over small masks: every candidate the filter drops leaves the next row empty
    rng = np.random.default_rng(0)
    for _ in range(20000):
        n = int(rng.integers(4, 12))
        mask = (1 << n) - 1
        nc = int(rng.integers(0, 1 << n)) & mask
        l = (int(rng.integers(0, 1 << n)) << 1) & 0xFFFFFFFF
        r = int(rng.integers(0, 1 << n)) >> 1
        a = nc & ~(l | r)
        kept = drop_leaves(a, nc, l, r)
        assert kept & ~a == 0
        for c in range(n):
            b = 1 << c
            if a & b and not kept & b:
                nxt = (nc - b) & ~((((l + b) << 1) & 0xFFFFFFFF) | ((r + b) >> 1))
                assert nxt == 0, (n, nc, l, r, c)
