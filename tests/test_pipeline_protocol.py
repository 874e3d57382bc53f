"""CPU model of the stage ring of the two-group TMA pass (k_pass_tma2).

Three shared-memory stages, one mbarrier each (arrival count 1 + the TMA
byte count); group g computes this CTA's tiles j = g, g+2, ...; tile j uses
stage j % 3 and waits for phase j // 3 by parity; when a group has read
tile j for the last time it issues tile j + 3 into the same stage.  A parity
wait cannot tell phase k from phase k - 2, so a group that reaches tile j
while the stage is still in tile j - 3's phase would pass at once and the
later refill would arrive twice on one phase.  The kernel therefore waits
for the stage's issued-tile index to reach j first.  The model checks that
the guarded protocol never waits on the wrong phase or arrives twice, and
that the unguarded one can.
"""
import heapq
import random


def simulate(guard, tiles=60, seed=0, load=(1.0, 12.0), comp=(0.5, 6.0)):
    rnd = random.Random(seed)
    S = 3
    completed = [0] * S      # completed phases per stage
    issued = [-1] * S        # last tile issued into each stage
    arrivals = [0] * S       # arrivals in the current phase
    events = []
    faults = []

    def issue(j, now):
        s = j % S
        issued[s] = j
        arrivals[s] += 1
        if arrivals[s] > 1:
            faults.append(("double arrive", s, j))
        heapq.heappush(events, (now + rnd.uniform(*load), "land", s, j))

    for j in range(min(S, tiles)):
        issue(j, 0.0)
    nxt = {0: 0, 1: 1}
    blocked = {0: True, 1: True}

    def try_start(g, now):
        j = nxt[g]
        if j >= tiles:
            blocked[g] = False
            return
        s = j % S
        if guard and issued[s] != j:
            blocked[g] = True
            return
        if (completed[s] & 1) != ((j // S) & 1):  # try_wait.parity returns true
            if completed[s] != j // S + 1 or issued[s] != j:
                faults.append(("wrong phase", g, j))
            blocked[g] = False
            heapq.heappush(events, (now + rnd.uniform(*comp), "done", g, j))
        else:
            blocked[g] = True

    for g in (0, 1):
        try_start(g, 0.0)
    while events and not faults:
        now, kind, a, b = heapq.heappop(events)
        if kind == "land":
            completed[a] += 1
            arrivals[a] = 0
        else:
            if b + S < tiles:
                issue(b + S, now)
            nxt[a] = b + 2
            blocked[a] = True
        for g in (0, 1):
            if blocked[g]:
                try_start(g, now)
    return faults


def test_guarded_ring_is_consistent():
    for seed in range(300):
        assert simulate(True, seed=seed) == []


def test_unguarded_ring_can_alias_phases():
    bad = sum(1 for seed in range(300) if simulate(False, seed=seed))
    assert bad > 0
