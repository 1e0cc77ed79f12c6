"""The set-aside rule of the trace kernel (run_ray with SKIP), restated as a
small host model and checked against the in-order rule on random cases.

A ray's candidates come in DFS order; each lies in a brick and either hits
or not.  In-order (the reference): the first hitting candidate decides the
pixel, and a ray waits a pass for each absent brick it reaches.  Set-aside:
up to K absent candidates are set aside per pass (their bricks requested)
while later resident candidates are marched; a hit past set-aside
candidates is tentative, and the next pass marches the set-aside ones
first.  The model follows the kernel's state machine step for step; the
property is that the pixel never differs and that passes never grow.
The GPU parity tests check the kernel itself against the oracle."""
import random


def in_order(cands, resident_at):
    """(hit index or None, passes): one absent brick discovered per pass"""
    passes, loaded = 1, set()
    for i, (brick, hit) in enumerate(cands):
        while brick not in loaded and not resident_at(brick, passes):
            loaded.add(brick)            # requested, serviced between passes
            passes += 1
        if hit:
            return i, passes
    return None, passes


def set_aside(cands, resident_at, K, evict=None, max_passes=1000):
    """the kernel's rule: returns (hit index or None, passes).  evict(loaded,
    requested, passes) -> bricks the service between passes drops again
    (never those it loads for this pass's requests, as the cache never
    evicts a slot stamped by the pass that follows)."""
    passes, loaded = 1, set()
    pos, aside, tent = 0, [], None
    resume = False

    def present(b):
        return b in loaded or resident_at(b, passes)

    while True:
        requested = set()
        suspended = False
        if resume:                       # set-aside candidates first, in order
            while aside:
                i = aside[0]
                b, hit = cands[i]
                if not present(b):
                    requested.add(b)
                    suspended = True
                    break
                aside.pop(0)
                if hit:
                    return i, passes     # earliest hit wins over a tentative one
            if not suspended:
                resume = False
                if tent is not None:
                    return tent, passes
        if not suspended:
            while pos < len(cands):
                b, hit = cands[pos]
                if not present(b):
                    requested.add(b)
                    if len(aside) < K:
                        aside.append(pos)
                        pos += 1
                        continue
                    suspended = True     # the candidate stays on the stack
                    break
                if hit:
                    if not aside:
                        return pos, passes
                    tent = pos           # tentative: the rest of the DFS is dropped
                    pos = len(cands)
                    suspended = True
                    break
                pos += 1
            else:
                if not aside:
                    return None, passes
                suspended = True
        if evict is not None:
            loaded -= evict(loaded - requested, requested, passes)
        loaded |= requested
        passes += 1
        assert passes <= max_passes, "no progress"
        resume = True


def test_set_aside_keeps_the_in_order_pixel_and_never_adds_passes():
    rng = random.Random(7)
    for _ in range(4000):
        n = rng.randint(0, 12)
        nbricks = rng.randint(1, 6)
        cands = [(rng.randrange(nbricks), rng.random() < 0.25) for _ in range(n)]
        warm = {b for b in range(nbricks) if rng.random() < 0.4}

        def resident_at(b, p, warm=warm):
            return b in warm
        want, p0 = in_order(cands, resident_at)
        for K in (1, 2, 4):
            got, p1 = set_aside(cands, resident_at, K)
            assert got == want, (cands, warm, K)
            assert p1 <= p0, (cands, warm, K)


def test_set_aside_keeps_the_in_order_pixel_when_bricks_are_evicted_between_passes():
    """Bricks loaded for earlier passes may be evicted again before the
    set-aside candidates are marched: the resumed candidate then finds its
    brick absent, requests it and suspends (the kernel's CAND_MISSING ->
    RAY_SUSPENDED in the resume loop).  The pixel is still the in-order
    one; the pass count may grow."""
    rng = random.Random(11)
    for _ in range(4000):
        n = rng.randint(0, 12)
        nbricks = rng.randint(1, 6)
        cands = [(rng.randrange(nbricks), rng.random() < 0.25) for _ in range(n)]
        warm = {b for b in range(nbricks) if rng.random() < 0.3}
        evict_p = rng.choice((0.2, 0.5, 0.9))
        # warm bricks are resident only in the first pass: later passes see
        # them only once loaded, and loaded bricks can be evicted
        def resident_at(b, p, warm=warm):
            return p == 1 and b in warm

        def evict(old, requested, p, evict_p=evict_p, r=rng):
            return {b for b in old if r.random() < evict_p}
        want = next((i for i, (_, hit) in enumerate(cands) if hit), None)
        for K in (1, 2, 4):
            got, _ = set_aside(cands, resident_at, K, evict=evict)
            assert got == want, (cands, warm, K, evict_p)
