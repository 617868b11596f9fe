"""The original leaf search's survivor queue (k_leaves_sh1 in shockhash_b200/csrc/shg_leaves.cu)
restated on the CPU: rounds of 32 lanes x SPL seeds, coverage survivors appended in seed order
(t-major ballots), pseudoforest tests 32 at a time once kSh1Drain survivors wait, the first passing
entry in queue order taken. It must return what the reference's sequential loop returns
(ShockHash.h:404-434): the smallest seed that passes both tests, or nothing within the cap."""
import numpy as np
import pytest

SPL, DRAIN = 2, 4


def sequential(cover, forest, cap):
    for x in range(cap):
        if cover[x] and forest[x]:
            return x
    return None


def queued(cover, forest, cap, drain=DRAIN, spl=SPL):
    """The kernel's control flow; cover/forest cover every seed the rounds may touch."""
    q, found = [], None

    def drain_queue():
        nonlocal q, found
        for q0 in range(0, len(q), 32):
            if found is not None:
                break
            chunk = q[q0:q0 + 32]
            passing = [off for off in chunk if forest[off]]  # lanes in order: the ballot's first set bit
            if passing:
                found = passing[0]
        q = []

    base = 0
    while base < cap and found is None:
        for t in range(spl):  # all lanes' x + 32 t before x + 32 (t + 1)
            q.extend(base + 32 * t + lane for lane in range(32) if cover[base + 32 * t + lane])
        assert len(q) < drain + 32 * spl + 1  # the queue's capacity in shared memory
        if len(q) >= drain:
            drain_queue()
        base += 32 * spl
    if found is None and q:
        drain_queue()
    return found


@pytest.mark.parametrize("seed", range(40))
@pytest.mark.parametrize("p_cover,p_forest", [(0.02, 0.05), (0.1, 0.3), (0.5, 0.02), (0.9, 0.9)])
def test_queue_returns_the_sequential_answer(seed, p_cover, p_forest):
    rng = np.random.default_rng(seed)
    cap = 64 * int(rng.integers(1, 60))
    span = cap + 64
    cover = rng.random(span) < p_cover
    forest = rng.random(span) < p_forest
    got, want = queued(cover, forest, cap), sequential(cover, forest, span)
    # the kernel reports a trial-limit error for an answer at or past the cap, as before the queue
    if want is None or want >= cap:
        assert got is None or got >= cap
    else:
        assert got == want


def test_edge_cases():
    span = 64 * 10
    none = np.zeros(span, bool)
    assert queued(none, none, 64 * 8) is None
    # survivors that all fail the pseudoforest test, then one that passes in the last drained chunk
    cover = np.zeros(span, bool)
    forest = np.zeros(span, bool)
    cover[:40] = True
    forest[39] = True
    assert queued(cover, forest, 64 * 8) == 39
    # a passing survivor that waits in a partly filled queue until the cap ends the rounds
    cover = np.zeros(span, bool)
    forest = np.zeros(span, bool)
    cover[200] = True
    forest[200] = True
    assert queued(cover, forest, 256) == 200
    # an earlier survivor that fails and a later one in the same drain that passes
    cover = np.zeros(span, bool)
    forest = np.zeros(span, bool)
    cover[[3, 70, 130, 131]] = True
    forest[[131]] = True
    assert queued(cover, forest, 64 * 9) == 131
