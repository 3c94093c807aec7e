"""The forward kernel's stage hand-over, replayed on the CPU.

Each CTA of `bp_mixed_kernel` runs 8 warps over two stage buffers with three
mbarriers per buffer (csrc/bp_mixed.cu):

* full[b]  -- one arrival per pulse slot (and the window bytes);
* ready[b] -- one arrival per warp once its window is in intercept form;
* empty[b] -- one arrival per warp once it has consumed the stage.

Per stage i (buffer s = i & 1) a warp: waits empty[s^1] for stage i - 1 and
produces stage i + 1 into buffer s^1; waits ready[s] for stage i; consumes
it and arrives on empty[s]; waits full[s^1] for stage i + 1, rewrites its
window and arrives on ready[s^1].  Every wait is a parity wait (the phase
with parity p has completed once the barrier's phase count has parity !p).

The model runs the 8 warp programs under random interleavings and checks
that no interleaving deadlocks, that every wait is released by the phase of
its own stage (never one stage early or late: a parity wait cannot tell
them apart), and that no warp overwrites a buffer another warp still reads.
"""
import random

import pytest

WARPS = 8


class Barrier:
    def __init__(self, count):
        self.count = count
        self.pending = count
        self.phases = 0  # completed phases

    def arrive(self):
        self.pending -= 1
        assert self.pending >= 0
        if self.pending == 0:
            self.phases += 1
            self.pending = self.count

    def passed(self, parity):
        return (self.phases & 1) != parity


def warp_program(n):
    """The kernel's per-warp sequence for n stages, as operations:
    ("wait", barrier, parity, (kind, stage)), ("arrive", barrier) and
    ("do", action, stage, buffer)."""
    yield ("do", "produce", 0, 0)
    yield ("arrive", ("full", 0))
    yield ("wait", ("full", 0), 0, ("full", 0))
    yield ("do", "rewrite", 0, 0)
    yield ("arrive", ("ready", 0))
    for i in range(n):
        s = i & 1
        if i + 1 < n:
            if i >= 1:
                yield ("wait", ("empty", s ^ 1), ((i - 1) >> 1) & 1, ("empty", i - 1))
            yield ("do", "produce", i + 1, s ^ 1)
            yield ("arrive", ("full", s ^ 1))
        yield ("wait", ("ready", s), (i >> 1) & 1, ("ready", i))
        yield ("do", "consume", i, s)
        yield ("arrive", ("empty", s))
        if i + 1 < n:
            yield ("wait", ("full", s ^ 1), ((i + 1) >> 1) & 1, ("full", i + 1))
            yield ("do", "rewrite", i + 1, s ^ 1)
            yield ("arrive", ("ready", s ^ 1))


def replay(n, seed, program=warp_program):
    rnd = random.Random(seed)
    bars = {(kind, b): Barrier(WARPS) for kind in ("full", "ready", "empty") for b in range(2)}
    done = {}       # (barrier kind, stage) -> warps whose action for it is done
    readers = {}    # stage -> warps that consumed it
    progs = [program(n) for _ in range(WARPS)]
    op = [next(p) for p in progs]
    live = set(range(WARPS))
    while live:
        ready = [w for w in live if op[w][0] != "wait" or bars[op[w][1]].passed(op[w][2])]
        assert ready, f"deadlock: n={n} seed={seed} {[op[w] for w in sorted(live)]}"
        w = rnd.choice(ready)
        kind = op[w][0]
        if kind == "wait":
            # released by its own stage's phase: every warp did the action
            assert done.get(op[w][3], 0) == WARPS, op[w]
        elif kind == "arrive":
            bars[op[w][1]].arrive()
        else:
            _, action, stage, _buf = op[w]
            if action == "produce" and stage >= 2:
                # buffer reuse: stage - 2 was consumed by every warp
                assert len(readers.get(stage - 2, ())) == WARPS, (w, stage)
            if action == "rewrite" and stage >= 2:
                assert len(readers.get(stage - 2, ())) == WARPS, (w, stage)
            if action == "consume":
                readers.setdefault(stage, set()).add(w)
            key = {"produce": "full", "rewrite": "ready", "consume": "empty"}[action]
            done[(key, stage)] = done.get((key, stage), 0) + 1
        try:
            op[w] = next(progs[w])
        except StopIteration:
            live.discard(w)
    assert all(len(readers[i]) == WARPS for i in range(n))


@pytest.mark.parametrize("n", [1, 2, 3, 4, 7, 12])
def test_stage_hand_over_is_deadlock_free_and_phase_exact(n):
    for seed in range(200):
        replay(n, seed)


def test_replay_catches_a_missing_empty_wait():
    """The check has teeth: without the empty wait a warp refills a buffer
    that another warp has not finished reading."""
    def without_empty_wait(n):
        for op in warp_program(n):
            if op[0] == "wait" and op[1][0] == "empty":
                continue
            yield op

    with pytest.raises(AssertionError):
        for seed in range(200):
            replay(6, seed, without_empty_wait)
