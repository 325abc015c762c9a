"""The shared-column grey cost kernel's work split and neighbour rule (lux_b200/csrc/cost.cu, k_cost_axis_v), restated
on the CPU.

A warp covers a run of 32·P - 2 pixels of a row, P pixels (slots) a lane; slots 0 and 1 of lane 0 are the two pixels left
of the run, computed for their block columns and never stored. A slot takes its block's middle and left columns from the
two pixels to its left when the neighbour rule says their targets are exactly 2 and 4 half-pixels to the left:
  * lane L's slot P-1 target goes to lane L+1 by shuffle, replaced by a sentinel unless slot P-2's target is one pixel
    left of it; lane 0 receives its own values (shfl_up);
  * fast[0] = tx[0] - t_left == 2, fast[1] = fast[0] and pair[1], fast[j] = pair[j] and pair[j-1] for j >= 2, with
    pair[j] = tx[j] - tx[j-1] == 2, all compares mod 2^32.
These tests check that the runs store every pixel of a row exactly once, and that wherever the rule holds for a stored
pixel inside the rect, its neighbours' targets are exactly the ones the block needs, for any target sequence.
"""
import os
import random
import re

import pytest

M32 = 0xFFFFFFFF
NO_ROW = -(1 << 31)
HERE = os.path.dirname(os.path.abspath(__file__))


def _kernel_px():
    src = open(os.path.join(HERE, "..", "lux_b200", "csrc", "cost.cu")).read()
    return int(re.search(r"constexpr int kAxPx = (\d+);", src).group(1))


def _runs(W, P):
    run = 32 * P - 2
    stored = []
    for r in range((W + run - 1) // run):
        x0 = r * run - 2
        for lane in range(32):
            for j in range(P):
                x = x0 + lane * P + j
                if lane * P + j >= 2 and x < W:
                    stored.append(x)
    return stored


@pytest.mark.parametrize("P", [2, 4])
def test_runs_store_every_pixel_once(P):
    for W in list(range(1, 300)) + [1040, 2080, 4159, 4160, 4161, 5216]:
        stored = _runs(W, P)
        assert sorted(stored) == list(range(W)), (P, W)


def test_kernel_px_is_covered():
    assert _kernel_px() in (2, 4)


def _fast_flags(tx, P):
    """tx: 32·P targets (int32) of one run, slot s = lane·P + j. Returns fast[s] and the slots that provide the middle
    and left columns of slot s under the kernel's rule."""
    n = 32 * P
    fast, mid, left = [False] * n, [None] * n, [None] * n

    def eq2(a, b):  # (a - b) mod 2^32 == 2
        return ((a - b) & M32) == 2

    for lane in range(32):
        t = tx[lane * P:(lane + 1) * P]
        src = lane - 1 if lane > 0 else lane  # shfl_up: lane 0 keeps its own values
        ts = tx[src * P:(src + 1) * P]
        t_left = ts[P - 1] if eq2(ts[P - 1], ts[P - 2]) else NO_ROW
        pair = [None] + [eq2(t[j], t[j - 1]) for j in range(1, P)]
        f = [eq2(t[0], t_left)]
        for j in range(1, P):
            f.append(pair[j] and (f[0] if j == 1 else pair[j - 1]))
        for j in range(P):
            s = lane * P + j
            fast[s] = f[j]
            ext = [src * P + P - 2, src * P + P - 1] + [lane * P + k for k in range(P)]
            left[s], mid[s] = ext[j], ext[j + 1]
    return fast, mid, left


@pytest.mark.parametrize("P", [2, 4])
def test_neighbour_rule_is_exact(P):
    rng = random.Random(P)
    extremes = [NO_ROW, NO_ROW + 2, (1 << 31) - 1, (1 << 31) - 3, -1, 0, 1, 2, 3]
    x1 = 200  # the rect's right bound: slots with 1 <= tx >> 1 < x1 are inside
    for trial in range(3000):
        n = 32 * P
        base = rng.randrange(-20, 400)
        kind = trial % 4
        tx = []
        for s in range(n):
            if kind == 0:  # a rectified pair: one pixel a step, with occasional jumps
                base += 2 if rng.random() < 0.9 else rng.choice([0, 1, 3, 4, -2])
            elif kind == 1:  # a wider focal length
                base += rng.choice([2, 3])
            elif kind == 2:  # a narrower one
                base += rng.choice([1, 2])
            else:  # anything, extremes included
                base = rng.choice(extremes) if rng.random() < 0.3 else rng.randrange(-50, 450)
            tx.append(((base + (1 << 31)) & M32) - (1 << 31))
        fast, mid, left = _fast_flags(tx, P)
        for s in range(2, n):  # stored slots
            ix = tx[s] >> 1
            if fast[s] and 1 <= ix < x1:
                assert tx[mid[s]] == tx[s] - 2 and tx[left[s]] == tx[s] - 4, (P, trial, s, tx[left[s]], tx[mid[s]], tx[s])
