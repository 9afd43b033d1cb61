"""Ticket schedule of the plane-chained passes (libgrid_b200/csrc/cuda/gb_plane.cuh,
k_chain), restated on the CPU.

Ticket tk decodes to group g = tk // (S * TILES), stage s = (tk % (S * TILES))
// TILES, tile = tk % TILES and plane p = g - s * lag; tickets whose plane
falls outside [0, nplanes) are empty.  The chain cannot deadlock because
every tile a stage-s tile waits for (the stage s - 1 tiles of its plane)
holds a smaller ticket, and tickets are only drawn by running CTAs.  These
tests check both facts and run a discrete-event model of R resident CTAs
that, like the kernel, draw their next ticket one tile ahead."""
import heapq
import random

import pytest


def decode(tk, S, TILES, lag):
    g, rem = divmod(tk, S * TILES)
    s, tile = divmod(rem, TILES)
    return s, tile, g - s * lag


def total_tickets(nplanes, S, TILES, lag):
    return (nplanes + (S - 1) * lag) * S * TILES


def chain_lag(resident, S, TILES, pct=200):
    group = S * TILES
    return (resident * pct // 100 + group - 1) // group


@pytest.mark.parametrize("nplanes", [2, 3, 16, 256])
@pytest.mark.parametrize("S", [2, 3])
def test_every_tile_once_and_dependencies_earlier(nplanes, S):
    TILES = 32
    lag = chain_lag(592, S, TILES)
    seen = {}
    for tk in range(total_tickets(nplanes, S, TILES, lag)):
        s, tile, p = decode(tk, S, TILES, lag)
        if 0 <= p < nplanes:
            assert (s, tile, p) not in seen
            seen[(s, tile, p)] = tk
    assert len(seen) == S * TILES * nplanes
    for (s, tile, p), tk in seen.items():
        if s > 0:
            assert max(seen[(s - 1, t, p)] for t in range(TILES)) < tk


def simulate(nplanes, S, TILES, lag, resident, seed):
    """Resident CTAs draw tickets in order (one tile ahead); a stage-s tile
    starts once all stage s - 1 tiles of its plane are done.  Returns the
    number of completed tiles; a deadlock leaves tiles undone."""
    rnd = random.Random(seed)
    total = total_tickets(nplanes, S, TILES, lag)
    nxt = 0
    done = {}
    waiting = []
    events = []

    def draw():
        nonlocal nxt
        tk = nxt
        nxt += 1
        return tk

    def start(cta, tk, now):
        """Begin ticket tk on cta (which already holds its next ticket)."""
        while tk < total:
            s, tile, p = decode(tk, S, TILES, lag)
            if 0 <= p < nplanes:
                if s > 0 and done.get((s - 1, p), 0) < TILES:
                    waiting.append((cta, tk))
                    return
                heapq.heappush(events, (now + rnd.uniform(1.0, 3.0), cta, tk))
                return
            # empty ticket: go on with the held one and draw the next ahead
            tk = held[cta]
            held[cta] = draw()

    held = {}
    for cta in range(resident):
        tk = draw()
        held[cta] = draw()  # drawn one tile ahead
        start(cta, tk, 0.0)
    completed = 0
    while events:
        now, cta, tk = heapq.heappop(events)
        s, tile, p = decode(tk, S, TILES, lag)
        done[(s, p)] = done.get((s, p), 0) + 1
        completed += 1
        still = []
        for c2, t2 in waiting:
            s2, _, p2 = decode(t2, S, TILES, lag)
            if done.get((s2 - 1, p2), 0) >= TILES:
                heapq.heappush(events, (now + rnd.uniform(1.0, 3.0), c2, t2))
            else:
                still.append((c2, t2))
        waiting[:] = still
        tk2 = held[cta]
        held[cta] = draw()
        start(cta, tk2, now)
    return completed, waiting


@pytest.mark.parametrize("nplanes", [2, 5, 64])
@pytest.mark.parametrize("S", [2, 3])
@pytest.mark.parametrize("resident", [1, 7, 148, 592])
def test_no_deadlock(nplanes, S, resident):
    TILES = 32
    lag = chain_lag(resident, S, TILES)
    completed, waiting = simulate(nplanes, S, TILES, lag, resident, seed=nplanes * 31 + S * 7 + resident)
    assert not waiting
    assert completed == S * TILES * nplanes
