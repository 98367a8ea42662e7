"""The planner of the one-launch batch form (scft_team_schedule), on the host alone.

The batch kernel runs every chain of every instance on a team of CTAs; each CTA works
through its own ordered task list, and the members of a team exchange data every contour
step, so a CTA that waits for a partner still busy with another task stalls.  These tests
check the plans the library makes: team sizes divide the grid side, every chain gets
exactly its team (distinct CTAs, ranks 0..T-1), and a simulation of the task lists (a
task runs when all its members have reached it) always completes, for the configured
batch and for random ones.
"""
import ctypes

import numpy as np
import pytest

from crysscft_sample_b200 import _lib, batch


def schedule(n, U, G, fixed=None):
    L = _lib.load()
    J = len(n)
    cn = (ctypes.c_int * J)(*n)
    cu = (ctypes.c_int * J)(*U)
    fixed = fixed or {}
    fs = (ctypes.c_int * max(1, len(fixed)))(*fixed.keys())
    fz = (ctypes.c_int * max(1, len(fixed)))(*fixed.values())
    size = (ctypes.c_int * J)()
    cap = sum(n) * 1 + 1  # at most one task per unit
    tc, tr, ts = (ctypes.c_int * cap)(), (ctypes.c_int * cap)(), (ctypes.c_int * cap)()
    tb = (ctypes.c_int * (G + 1))()
    nt = ctypes.c_size_t()
    pl, lb = ctypes.c_double(), ctypes.c_double()
    _lib.check(L.scft_team_schedule(J, cn, cu, G, len(fixed), fs, fz, size, cap, tc, tr, ts, tb, ctypes.byref(nt),
                                    ctypes.byref(pl), ctypes.byref(lb)))
    k = nt.value
    tasks = [(tc[t], tr[t], ts[t]) for t in range(k)]
    begin = [tb[b] for b in range(G + 1)]
    return list(size), tasks, begin, pl.value, lb.value


def check_plan(n, size, tasks, begin, G):
    """Team sizes divide the grid sides; each chain has its ranks on distinct CTAs."""
    J = len(n)
    assert begin[0] == 0 and begin[-1] == len(tasks)
    assert all(begin[b] <= begin[b + 1] for b in range(G))
    members = {j: [] for j in range(J)}
    for b in range(G):
        for t in range(begin[b], begin[b + 1]):
            c, r, s = tasks[t]
            assert s == size[c]
            members[c].append((b, r))
    for j in range(J):
        T = size[j]
        assert 1 <= T <= min(n[j], G) and n[j] % T == 0
        ctas = [b for b, _ in members[j]]
        ranks = sorted(r for _, r in members[j])
        assert ranks == list(range(T)), f"chain {j}: ranks {ranks}"
        assert len(set(ctas)) == T, f"chain {j}: a CTA holds two ranks of one team"
        # the units rank, rank + T, ... of all ranks cover 0..n-1 once
        units = sorted(r + i * T for r in range(T) for i in range(n[j] // T))
        assert units == list(range(n[j]))


def simulate(tasks, begin, G):
    """Run the task lists: a task advances when every member CTA is at it.  True if all finish."""
    pos = [begin[b] for b in range(G)]
    at = {}
    for b in range(G):
        if pos[b] < begin[b + 1]:
            at.setdefault(tasks[pos[b]][0], set()).add(b)
    done = 0
    total = len(tasks)
    progress = True
    while progress:
        progress = False
        for c in list(at):
            members = at[c]
            size = tasks[pos[next(iter(members))]][2]
            if len(members) == size:
                del at[c]
                for b in members:
                    pos[b] += 1
                    done += 1
                    if pos[b] < begin[b + 1]:
                        at.setdefault(tasks[pos[b]][0], set()).add(b)
                progress = True
    return done == total


@pytest.mark.parametrize("fixed", [None, {16: 1, 24: 1, 32: 1, 48: 1, 64: 1}, {64: 32, 48: 24}])
def test_configured_batch_plan_is_complete_and_cannot_deadlock(fixed):
    cfg = batch.batch_config(64)
    ds = 0.01
    n, U = [], []
    for c in cfg:
        for _ in range(2):  # forward and backward chain
            n.append(c["N"][0] // 2)
            U.append(int(c["fA"] / ds) + int((1 - c["fA"]) / ds))
    G = 148
    size, tasks, begin, planned, bound = schedule(n, U, G, fixed)
    check_plan(n, size, tasks, begin, G)
    for j, side in enumerate(n):
        if fixed and side in fixed:
            assert size[j] == fixed[side]
    assert simulate(tasks, begin, G)
    assert bound <= planned
    if fixed is None:  # the planner's own choice packs within 15 % of the lower bound
        assert planned < 1.15 * bound, (planned, bound)


def test_planner_prefers_small_teams_when_the_cost_model_allows():
    # one chain per side on many CTAs: every chain can run alone on the widest team; the
    # planner takes the team size that fits the makespan with the fewest CTAs
    n, U = [64, 64], [100, 100]
    size, tasks, begin, planned, bound = schedule(n, U, 148)
    assert size[0] == size[1] and 64 % size[0] == 0
    size_small, *_ = schedule(n * 40, U * 40, 148)
    assert max(size_small) <= size[0]


def test_random_plans_cannot_deadlock():
    rng = np.random.default_rng(5)
    for trial in range(200):
        J = int(rng.integers(1, 40))
        n = [int(8 * rng.integers(1, 9)) for _ in range(J)]
        U = [int(rng.integers(1, 300)) for _ in range(J)]
        G = int(rng.integers(len(set(n)), 149))
        size, tasks, begin, _, _ = schedule(n, U, G)
        check_plan(n, size, tasks, begin, G)
        assert simulate(tasks, begin, G), f"trial {trial}: plan stalls"


def test_schedule_rejects_bad_arguments():
    L = _lib.load()
    one = (ctypes.c_int * 1)(16)
    three = (ctypes.c_int * 1)(3)
    size = (ctypes.c_int * 1)()
    tb = (ctypes.c_int * 2)()
    nt = ctypes.c_size_t()
    t = (ctypes.c_int * 16)()
    assert L.scft_team_schedule(1, one, one, 0, 0, None, None, size, 16, t, t, t, tb, ctypes.byref(nt), None, None) != 0
    # a fixed team size that does not divide the grid side
    assert L.scft_team_schedule(1, one, one, 4, 1, one, three, size, 16, t, t, t, tb, ctypes.byref(nt), None,
                                None) != 0
    # too little room for the tasks
    assert L.scft_team_schedule(1, one, one, 1, 0, None, None, size, 0, t, t, t, tb, ctypes.byref(nt), None, None) != 0
    assert nt.value == 1
