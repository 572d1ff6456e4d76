"""Host model of the blind rotation's key-row ring without a producer warp (blind_rotate.cu,
blind_rotate_kernel with PW = false): G teams consume rows 0..R-1 in order from a D-slot ring; row r
may enter slot r % D only after every team has released row r - D.  Thread 0 (a thread of team 0)
issues the first D rows at the start; before waiting for row c it issues, blocking on the slot, every
row up to c not yet issued; after releasing a row it issues further rows while their slots test free.

The model runs teams at random speeds and checks that every run ends (no deadlock: a team never
waits for a row nobody will issue) and that no row is copied into a slot still held.  Failure detection of the real kernel (bounded waits) is tested on the GPU;
this covers the protocol itself on the CPU."""
import numpy as np
import pytest


def simulate(G, D, R, rng, latency=3, slow0=1, issue_before_wait=True):
    # per team: next row to consume, remaining work on the current row (None = waiting for it)
    nxt = [0] * G
    work = [None] * G
    released = np.zeros(R, dtype=np.int32)  # teams that released each row
    arrive = {}                              # row -> time its copy lands
    issued = 0
    slot_row = [-1] * D                      # row whose copy occupies each slot
    t0_blocked = False                       # thread 0 blocked issuing (its team waits)

    def slot_free(r):
        return r < D or released[r - D] == G

    def issue(r, now):
        nonlocal issued
        assert slot_free(r), "row copied into a slot still held"
        prev = slot_row[r % D]
        assert prev == -1 or prev == r - D
        slot_row[r % D] = r
        arrive[r] = now + latency
        issued = r + 1

    while issued < min(D, R):
        issue(issued, 0)
    now = 0
    idle_steps = 0
    while min(nxt) < R:
        now += 1
        progressed = False
        for g in rng.permutation(G):
            if nxt[g] >= R:
                continue
            if work[g] is None:
                c = nxt[g]
                if g == 0 and issue_before_wait:
                    # thread 0 issues every row up to c before waiting for it (blocking on slots)
                    t0_blocked = False
                    while issued <= c and issued < R:
                        if not slot_free(issued):
                            t0_blocked = True
                            break
                        issue(issued, now)
                        progressed = True
                    if t0_blocked:
                        continue
                if c < issued and arrive[c] <= now:
                    work[g] = int(rng.integers(1, 6)) * (slow0 if g == 0 else 1)
                    progressed = True
                continue
            work[g] -= 1
            progressed = True
            if work[g] == 0:
                c = nxt[g]
                released[c] += 1
                nxt[g] += 1
                work[g] = None
                if g == 0:
                    while issued < R and slot_free(issued):
                        issue(issued, now)
        idle_steps = 0 if progressed else idle_steps + 1
        # copies in flight count as progress; anything longer than the latency is a deadlock
        assert idle_steps <= latency + 1, f"deadlock at rows {nxt}, issued {issued}"
    assert issued == R and (released == G).all()
    return now


@pytest.mark.parametrize("G,D", [(4, 4), (4, 6), (2, 3), (2, 4), (1, 4), (7, 6)])
def test_ring_without_producer_warp_never_deadlocks(G, D):
    rng = np.random.default_rng(100 * G + D)
    for trial in range(30):
        R = int(rng.integers(1, 60))
        simulate(G, D, R, rng)


def test_ring_with_a_slow_issuing_team():
    # team 0 (the issuer) 8x slower than the others: they wait on rows it issues late, but the run ends
    rng = np.random.default_rng(7)
    simulate(4, 4, 200, rng, latency=10, slow0=8)


def test_model_detects_a_protocol_that_deadlocks():
    # planted mistake, in the model: thread 0 only refills after releasing a row and never issues
    # before waiting.  Once team 0 runs ahead of a slot's last reader, it stops refilling, and
    # every team ends up waiting for a row that no one issues.
    rng = np.random.default_rng(3)
    with pytest.raises(AssertionError, match="deadlock"):
        for trial in range(50):
            simulate(4, 4, 60, rng, issue_before_wait=False)
