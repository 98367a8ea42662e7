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


def schedule(n, U, G, balance=1.0):
    L = _lib.load()
    J = len(n)
    cn = (ctypes.c_int * J)(*n)
    cu = (ctypes.c_int * J)(*U)
    size = (ctypes.c_int * J)()
    cap = sum(n) * 1 + 1  # at most one task per unit
    tc, tr, ts = (ctypes.c_int * cap)(), (ctypes.c_int * cap)(), (ctypes.c_int * cap)()
    tb = (ctypes.c_int * (G + 1))()
    nt = ctypes.c_size_t()
    pl, lb = ctypes.c_double(), ctypes.c_double()
    _lib.check(L.scft_team_schedule(J, cn, cu, G, float(balance), size, cap, tc, tr, ts, tb, ctypes.byref(nt),
                                    ctypes.byref(pl), ctypes.byref(lb)))
    k = nt.value
    tasks = [(tc[t], tr[t], ts[t]) for t in range(k)]
    begin = [tb[b] for b in range(G + 1)]
    return list(size), tasks, begin, pl.value, lb.value


def check_plan(n, size, tasks, begin, G):
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


@pytest.mark.parametrize("balance", [0.5, 1.0, 2.0])
def test_configured_batch_plan_is_complete_and_cannot_deadlock(balance):
    cfg = batch.batch_config(64)
    ds = 0.01
    n, U = [], []
    for c in cfg:
        for _ in range(2):  # forward and backward chain
            n.append(c["N"][0] // 2)
            U.append(int(c["fA"] / ds) + int((1 - c["fA"]) / ds))
    G = 148
    size, tasks, begin, planned, bound = schedule(n, U, G, balance)
    check_plan(n, size, tasks, begin, G)
    assert simulate(tasks, begin, G)
    assert bound <= planned < 2.0 * bound, (planned, bound)


def test_random_plans_cannot_deadlock():
    rng = np.random.default_rng(5)
    for trial in range(200):
        J = int(rng.integers(1, 40))
        n = [int(8 * rng.integers(1, 9)) for _ in range(J)]
        U = [int(rng.integers(1, 300)) for _ in range(J)]
        G = int(rng.integers(1, 149))
        balance = float(rng.choice([0.25, 0.5, 1.0, 2.0, 4.0]))
        size, tasks, begin, _, _ = schedule(n, U, G, balance)
        check_plan(n, size, tasks, begin, G)
        assert simulate(tasks, begin, G), f"trial {trial}: plan stalls"


def test_schedule_rejects_bad_arguments():
    L = _lib.load()
    one = (ctypes.c_int * 1)(16)
    size = (ctypes.c_int * 1)()
    tb = (ctypes.c_int * 2)()
    nt = ctypes.c_size_t()
    t = (ctypes.c_int * 16)()
    assert L.scft_team_schedule(1, one, one, 0, 1.0, size, 16, t, t, t, tb, ctypes.byref(nt), None, None) != 0
    assert L.scft_team_schedule(1, one, one, 1, 0.0, size, 16, t, t, t, tb, ctypes.byref(nt), None, None) != 0
    # too little room for the tasks
    assert L.scft_team_schedule(1, one, one, 1, 1.0, size, 0, t, t, t, tb, ctypes.byref(nt), None, None) != 0
    assert nt.value == 1
