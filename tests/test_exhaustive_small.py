"""Exhaustive safety on small instances (the reference's tests/exhaustive/check_small_instances.py
idea, restated): for n = 6..12 seeded complete EUC_2D graphs, every edge the JV fixed-point loop
deletes must lie on no optimal tour. The set of all optimal-tour edges comes from a Held-Karp
dynamic program that keeps every optimal predecessor. The CPU oracle runs the loop; the GPU test
runs the same loop with the B200 screen in place of the CPU screen."""
import random

import numpy as np
import pytest

from helpers import commit, complete_graph


def euc(a, b):
    import math
    s = (a[0] - b[0]) ** 2 + (a[1] - b[1]) ** 2
    r = math.isqrt(s)
    return r + (1 if s - r * r > r else 0)


def instance(n):
    rng = random.Random(0xC0DA0000 + n)
    points = []
    while len(points) < n:
        p = (rng.randrange(0, 2001), rng.randrange(0, 2001))
        if p not in points:
            points.append(p)
    return points


def optimal_edges(points):
    n = len(points)
    d = [[euc(points[u], points[v]) for v in range(n)] for u in range(n)]
    dp, pred = {}, {}
    for last in range(1, n):
        dp[1 << last, last] = d[0][last]
        pred[1 << last, last] = [0]
    for size in range(2, n):
        for mask in range(1 << n):
            if mask & 1 or bin(mask).count("1") != size:
                continue
            for last in range(1, n):
                if not mask >> last & 1:
                    continue
                prev_mask = mask ^ (1 << last)
                best, preds = None, []
                for prev in range(1, n):
                    if prev_mask >> prev & 1:
                        value = dp[prev_mask, prev] + d[prev][last]
                        if best is None or value < best:
                            best, preds = value, [prev]
                        elif value == best:
                            preds.append(prev)
                dp[mask, last], pred[mask, last] = best, preds
    full = ((1 << n) - 1) ^ 1
    optimum = min(dp[full, last] + d[last][0] for last in range(1, n))
    edges, seen = set(), set()

    def back(mask, last):
        if (mask, last) in seen:
            return
        seen.add((mask, last))
        for prev in pred[mask, last]:
            edges.add((min(prev, last), max(prev, last)))
            if prev != 0:
                back(mask ^ (1 << last), prev)

    for last in range(1, n):
        if dp[full, last] + d[last][0] == optimum:
            edges.add((0, last))
            back(full, last)
    return edges


def removed_edges(g, final_active):
    return {(int(g.edge_u[e]), int(g.edge_v[e])) for e in np.flatnonzero(final_active == 0)}


def test_oracle_never_deletes_an_optimal_edge(port):
    total = 0
    for n in range(6, 13):
        pts = instance(n)
        g = complete_graph([p[0] for p in pts], [p[1] for p in pts])
        active, _, _, _ = port.jv_eliminate(g)
        removed = removed_edges(g, active)
        assert not (removed & optimal_edges(pts)), n
        total += len(removed)
    assert total > 0  # the instances do exercise deletions


@pytest.mark.gpu
def test_gpu_screen_never_deletes_an_optimal_edge(ctx, port):
    for n in range(6, 13):
        pts = instance(n)
        g = complete_graph([p[0] for p in pts], [p[1] for p in pts])
        start = g
        while True:
            witness, _ = ctx.jv_screen(g)
            np.testing.assert_array_equal(witness, port.jv_screen(g))
            g, committed = commit(port, g, witness)
            if committed == 0:
                break
        assert not (removed_edges(start, g.active) & optimal_edges(pts)), n
