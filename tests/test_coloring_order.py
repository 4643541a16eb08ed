"""The round-by-round order the preparation kernel colors and levels contacts in (visitInBodyOrder,
twofold_b200/csrc/tf_kernels.cuh), restated in Python: in each round every pending contact that is the first
pending one at each of its moving bodies is visited, and after a fixed number of rounds the rest are visited in
list order (also once a round visits fewer entries than a threshold). Greedy colors (src/lanes.cpp:356-374) and
levels computed in that order must equal the ones a single pass in list order computes, on random contact
lists, on long chains that outlast the rounds, and with contacts that take no color."""
import numpy as np
import pytest

NONE = -1
ROUNDS = 64


def greedy_sequential(ends, colorable):
    masks = {}
    out = []
    for (a, b), ok in zip(ends, colorable):
        if not ok:
            out.append(32)
            continue
        taken = (masks.get(a, 0) if a != NONE else 0) | (masks.get(b, 0) if b != NONE else 0)
        if taken == 0xFFFFFFFF:
            out.append(32)
            continue
        f = (~taken & (taken + 1)).bit_length() - 1
        for e in (a, b):
            if e != NONE:
                masks[e] = masks.get(e, 0) | (1 << f)
        out.append(f)
    return out


def levels_sequential(ends):
    last, out = {}, []
    for a, b in ends:
        lev = max(last.get(a, 0) if a != NONE else 0, last.get(b, 0) if b != NONE else 0)
        for e in (a, b):
            if e != NONE:
                last[e] = lev + 1
        out.append(lev)
    return out


def in_body_order(ends, pending, visit, rounds=ROUNDS, worth=0):
    """Calls visit on every pending entry in the order visitInBodyOrder does, checking that the entries of a
    round share no body."""
    n = len(ends)
    for _ in range(rounds):
        first = {}
        left = [x for x in range(n) if pending(x)]
        if not left:
            return
        for x in left:
            for e in ends[x]:
                if e != NONE:
                    first[e] = min(first.get(e, n), x)
        ready = [x for x in left if all(e == NONE or first[e] == x for e in ends[x])]
        seen = set()
        for x in ready:  # entries of one round share no body
            for e in ends[x]:
                if e != NONE:
                    assert e not in seen
                    seen.add(e)
        for x in ready:
            visit(x)
        if len(ready) < worth:
            break
    for x in range(n):
        if pending(x):
            visit(x)


def greedy_rounds(ends, colorable, rounds=ROUNDS, worth=0):
    color = [None if ok else 32 for ok in colorable]
    masks = {}

    def visit(x):
        a, b = ends[x]
        taken = (masks.get(a, 0) if a != NONE else 0) | (masks.get(b, 0) if b != NONE else 0)
        if taken == 0xFFFFFFFF:
            color[x] = 32
            return
        f = (~taken & (taken + 1)).bit_length() - 1
        for e in (a, b):
            if e != NONE:
                masks[e] = masks.get(e, 0) | (1 << f)
        color[x] = f

    in_body_order(ends, lambda x: color[x] is None, visit, rounds, worth)
    return color


def levels_rounds(ends, rounds=ROUNDS, worth=0):
    level = [None] * len(ends)
    last = {}

    def visit(x):
        a, b = ends[x]
        lev = max(last.get(a, 0) if a != NONE else 0, last.get(b, 0) if b != NONE else 0)
        for e in (a, b):
            if e != NONE:
                last[e] = lev + 1
        level[x] = lev

    in_body_order(ends, lambda x: level[x] is None, visit, rounds, worth)
    return level


def random_ends(rng, n, bodies, p_static):
    ends = []
    for _ in range(n):
        a, b = rng.choice(bodies, 2, replace=False)
        a = NONE if rng.random() < p_static else int(a)
        b = NONE if rng.random() < p_static / 4 else int(b)
        ends.append((a, b))
    return ends


@pytest.mark.parametrize("seed", range(8))
def test_rounds_color_like_the_list_order_pass(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(64, 600))
    ends = random_ends(rng, n, int(rng.integers(8, 200)), 0.3)
    colorable = list(rng.random(n) > 0.1)
    assert greedy_rounds(ends, colorable) == greedy_sequential(ends, colorable)
    assert levels_rounds(ends) == levels_sequential(ends)
    assert greedy_rounds(ends, colorable, worth=8) == greedy_sequential(ends, colorable)
    assert levels_rounds(ends, worth=8) == levels_sequential(ends)


def test_chains_longer_than_the_rounds_finish_in_list_order():
    # A stack: contact k joins bodies k and k + 1, so contact k waits for contact k - 1; 300 rounds' worth.
    ends = [(k, k + 1) for k in range(300)] + [(NONE, k) for k in range(0, 300, 7)]
    colorable = [True] * len(ends)
    assert greedy_rounds(ends, colorable) == greedy_sequential(ends, colorable)
    assert levels_rounds(ends) == levels_sequential(ends)
    assert greedy_rounds(ends, colorable, rounds=3) == greedy_sequential(ends, colorable)


def test_a_body_with_more_than_32_contacts_runs_out_of_colors_alike():
    ends = [(0, k) for k in range(1, 80)] + [(k, k + 1) for k in range(1, 40)]
    colorable = [True] * len(ends)
    seq = greedy_sequential(ends, colorable)
    assert seq.count(32) > 0
    assert greedy_rounds(ends, colorable) == seq
