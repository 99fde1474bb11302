"""Host model of the strip-team hand-over (sw_pass with TEAM, k_strips).

The W warps of a team take the strips of one item round robin.  Strip s
writes its boundary column into buffer s % W (lane 31 writes rows t0-31..t0
in the block of steps starting at t0) and, after each block, publishes
(s << 16) | min(t0 + 1, rows) in its warp's progress word.  Strip s + 1 reads
rows [0, 2L) before its first block and rows [t0 + L, t0 + 2L) at the start
of block t0 > 0, each time after waiting until the previous warp published
that many rows of strip s.

This model runs those rules under random interleavings of the warps (a
warp advances one block at a time, whenever its wait is satisfied) and
checks the two properties the kernel relies on:
  * every boundary row a strip reads holds the value its own predecessor
    strip wrote (buffer s % W is never overwritten by strip s + W before
    strip s + 1 read it), and
  * no interleaving deadlocks (some warp can always advance until all
    strips are done).
"""
import random

import pytest

L = 32  # lanes of a team warp (LANES)


def _warp_program(w, warps, strips, rows, log):
    """Generator of warp w: yields ("wait", s, need) before a read that needs
    `need` published rows of strip s, and ("block",) after each block."""
    nsteps = rows + L - 1
    for s in range(w, strips, warps):
        has_in, has_out = s > 0, s + 1 < strips
        if has_in:
            yield ("wait", s - 1, min(2 * L, rows))
            log.append(("read", s, 0, min(2 * L, rows)))
        for t0 in range(0, nsteps, L):
            if has_in and t0 > 0:
                yield ("wait", s - 1, min(t0 + 2 * L, rows))
                log.append(("read", s, min(t0 + L, rows), min(t0 + 2 * L, rows)))
            if has_out:
                log.append(("write", s, max(t0 - (L - 1), 0), min(t0 + 1, rows)))
                log.append(("publish", s, min(t0 + 1, rows)))
            yield ("block",)


def _run(warps, strips, rows, rng, program=None):
    """One random interleaving of the warps running `program` (default: the
    kernel's rules); returns the number of scheduling rounds."""
    program = program or _warp_program
    buf = [[None] * rows for _ in range(warps)]  # strip whose value each row holds
    prog = [-1] * warps
    logs = [[] for _ in range(warps)]
    progs = [program(w, warps, strips, rows, logs[w]) for w in range(warps)]
    pending = [None] * warps  # the wait each warp is blocked on
    done = [False] * warps

    def apply(w):
        for ev in logs[w]:
            kind, s = ev[0], ev[1]
            if kind == "read":
                for r in range(ev[2], ev[3]):
                    assert buf[(s - 1) % warps][r] == s - 1, (
                        "strip %d read row %d of buffer %d holding strip %s" % (
                            s, r, (s - 1) % warps, buf[(s - 1) % warps][r]))
            elif kind == "write":
                for r in range(ev[2], ev[3]):
                    buf[s % warps][r] = s
            else:
                value = (s << 16) | ev[2]
                assert value >= prog[w], "progress word went down"
                prog[w] = value
        logs[w].clear()

    def step(w):
        """Advances warp w to its next wait or block end."""
        while True:
            try:
                ev = next(progs[w])
            except StopIteration:
                apply(w)
                done[w] = True
                return
            if ev[0] == "wait":
                pending[w] = ev
                apply(w)
                return
            apply(w)
            if rng.random() < 0.5:
                return  # yield the scheduler after a block

    def ready(w):
        ev = pending[w]
        if ev is None:
            return True
        _, s, need = ev
        return prog[(w - 1) % warps] >= ((s << 16) | need)

    rounds = 0
    while not all(done):
        runnable = [w for w in range(warps) if not done[w] and ready(w)]
        assert runnable, "deadlock: every unfinished warp waits (progress %s)" % prog
        w = rng.choice(runnable)
        pending[w] = None
        step(w)
        rounds += 1
    return rounds


@pytest.mark.parametrize("warps", [2, 3, 5, 8])
def test_hand_over_under_random_interleavings(warps):
    rng = random.Random(1000 + warps)
    for trial in range(60):
        strips = rng.randint(1, 3 * warps + 2)
        rows = rng.choice([1, 5, 31, 32, 33, 63, 64, 65, 100, 200, 257])
        _run(warps, strips, rows, rng)


def test_a_planted_early_overwrite_is_caught():
    """The model's check is live: a warp that ignores its waits reads rows
    its predecessor has not written yet and overwrites rows its successor
    has not read, and the read check fails."""
    rng = random.Random(7)

    def unguarded(w, warps, strips, rows, log):
        for ev in _warp_program(w, warps, strips, rows, log):
            if ev[0] == "wait" and w == 0:
                continue  # warp 0 runs without waiting (a broken protocol)
            yield ev

    with pytest.raises(AssertionError):
        for _ in range(50):
            _run(2, 6, 200, rng, unguarded)
