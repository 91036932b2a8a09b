"""A step-by-step model of the persistent engine's work scheduling
(begputhinning_b200/csrc/kernels.cu: engine_kernel, next_wave, produce,
wait_ticket, poll_ticket), run under random interleavings of the CTAs to
check the protocol itself: every wave's tiles are processed exactly once and
in pass order, no CTA waits forever, and every instance retires.  It
models the parts whose correctness does not depend on the thinning rule:
the two rings of tickets (ring 0 first), multiple bulk-ring tickets per
claim held across tiles, the one-look staging of a held ticket during the
bookkeeping, 3D gangs with their grid budget, and abandonment of tickets
left behind when a ring's last instance retires.  Wave sizes come from a
seeded script per instance instead of from tile changes."""
import random

import pytest

MAX_CLAIM = 4
GANG_MAX = 6


class Inst:
    def __init__(self, rng, dims):
        self.dims = dims
        self.prio = 0 if dims == 3 else 1
        if dims == 2:
            self.waves = [rng.randint(1, 9) for _ in range(rng.randint(1, 6))]
        else:
            self.waves = []
            for _ in range(rng.randint(1, 3)):  # iterations: union pass + five passes on its list
                self.waves += [rng.randint(1, 10)] * 6
        self.waves.append(0)  # the wave after the last holds no tile: retire
        self.done = 0
        self.gang = 0
        self.retired = False
        self.seen = {}  # pass -> tiles processed


class Model:
    def __init__(self, rng, insts, grid):
        self.rng = rng
        self.insts = insts
        self.grid = grid
        self.head = [0, 0]
        self.tail = [0, 0]
        self.items = [{}, {}]  # ticket -> (inst, tile, pass, n, gang)
        self.live = 0
        self.live_prio = [0, 0]
        self.budget = grid
        self.budget0 = self.budget
        self.producing = []  # pending item publications: (ring, ticket, item)
        self.eager_claim = False
        self.held_first = True

    def next_wave(self, ii, q1):
        """The wave of pass q1 of instance ii: reserve its tickets at once
        (the items appear one step at a time), or retire the instance."""
        inst = self.insts[ii]
        n = inst.waves[q1]
        if n == 0:
            inst.retired = True
            self.live_prio[inst.prio] -= 1
            self.live -= 1
            return
        inst.done = 0
        gang = False
        if inst.dims == 3 and q1 % 6 != 5 and n <= GANG_MAX and self.budget >= n:
            self.budget -= n
            inst.gang = 0
            gang = True
        r = inst.prio
        t0 = self.tail[r]
        self.tail[r] += n
        for i in range(n):
            self.producing.append((r, t0 + i, (ii, i, q1, n, gang)))

    def publish_one(self):
        if not self.producing:
            return False
        k = self.rng.randrange(len(self.producing))
        r, t, it = self.producing.pop(k)
        self.items[r][t] = it
        return True


class CTA:
    def __init__(self, m):
        self.m = m
        self.state = "claim"
        self.item = None
        self.cont = False
        self.ngot = None
        self.pend = 0
        self.pend_t = 0
        self.gpass = 0
        self.ticket = None
        self.take = None
        self.eager = None
        self.finished = False
        self.held_first = m.held_first

    def depth(self, r):
        return self.m.tail[r] - self.m.head[r]

    def step(self):
        """One atomic action; returns True when something changed."""
        m = self.m
        if self.state == "claim":
            if self.cont:
                self.state = "tile"
                return True
            if self.ngot is not None:
                self.item, self.ngot = self.ngot, None
                self.gpass = 0
                self.state = "tile"
                return True
            # the counters are read in one step and the fetch-and-add happens in
            # a later one, so other CTAs may take tickets in between (a ticket
            # can then lie past the tail and wait for a later wave)
            d0, d1 = self.depth(0), self.depth(1)
            # the engine consumes its held bulk tickets before taking a ring-0
            # ticket, so a CTA never joins a gang while it holds tickets that
            # other instances' waves wait for (held_first = False models the
            # earlier rule, which let ring 0 jump ahead of held tickets)
            ring0_waiting = self.pend > 0 and d0 > 0 and not self.held_first
            if self.pend > 0 and not ring0_waiting:
                self.ticket = (1, self.pend_t)
                self.pend -= 1
                self.pend_t += 1
                self.state = "wait"
                return True
            if ring0_waiting or d0 > 0:
                self.take = (0, 1)
            elif d1 >= 2 * m.grid:
                self.take = (1, min(MAX_CLAIM, d1 // m.grid))
            elif d1 > 0:
                self.take = (1, 1)
            else:
                if m.live == 0:
                    self.finished = True
                    self.state = "exit"
                    return True
                return False
            self.state = "take"
            return True
        if self.state == "take":
            r, k = self.take
            self.ticket = (r, m.head[r])
            m.head[r] += k
            if k > 1:
                self.pend = k - 1
                self.pend_t = self.ticket[1] + 1
            self.state = "wait"
            return True
        if self.state == "wait":
            r, t = self.ticket
            if t in m.items[r]:
                self.item = m.items[r].pop(t)
                self.gpass = 0
                self.state = "tile"
                return True
            if m.live_prio[r] == 0 and t >= m.tail[r]:  # abandoned
                self.state = "claim"
                return True
            return False
        if self.state == "tile":
            ii, tile, q, n, gang = self.item
            inst = m.insts[ii]
            assert not inst.retired
            assert q == len(inst.seen) - 1 or q == len(inst.seen), "passes out of order"
            inst.seen.setdefault(q, []).append(tile)
            assert inst.seen[q].count(tile) == 1, "tile processed twice in one pass"
            # thread 32: one look at the next held ticket
            if self.pend > 0 and not (gang and q % 6 != 5) and (self.held_first or self.depth(0) <= 0):
                if self.pend_t in m.items[1]:
                    self.ngot = m.items[1].pop(self.pend_t)
                    self.pend -= 1
                    self.pend_t += 1
            if m.eager_claim and self.depth(1) > 0 and not (gang and q % 6 != 5):
                # the dropped design: take a new ticket now and wait for its
                # item before recording this tile (and publishing its wave)
                self.eager = (1, m.head[1])
                m.head[1] += 1
                self.state = "eager"
                return True
            return self.finish_tile()
        if self.state == "eager":
            r, t = self.eager
            if t in m.items[r]:
                self.ngot = m.items[r].pop(t)
            elif not (m.live_prio[r] == 0 and t >= m.tail[r]):
                return False
            return self.finish_tile()
        if self.state == "gang":
            ii, tile, q, n, gang = self.item
            if m.insts[ii].gang >= n * self.gpass:
                self.item = (ii, tile, q + 1, n, gang)
                self.cont = True
                self.state = "claim"
                return True
            return False
        return False

    def finish_tile(self):
        m = self.m
        ii, tile, q, n, gang = self.item
        inst = m.insts[ii]
        self.cont = False
        if gang and q % 6 != 5:
            inst.gang += 1
            self.gpass += 1
            self.state = "gang"
            return True
        inst.done += 1
        last = inst.done == n
        if last and gang:
            m.budget += n
        if last:
            assert sorted(inst.seen[q]) == list(range(n))
            m.next_wave(ii, q + 1)
        self.state = "claim"
        return True


def run_model(seed, grid, n2d, n3d, eager_claim=False, budget=None):
    rng = random.Random(seed)
    insts = [Inst(rng, 2) for _ in range(n2d)] + [Inst(rng, 3) for _ in range(n3d)]
    rng.shuffle(insts)
    m = Model(rng, insts, grid)
    m.eager_claim = eager_claim
    if budget is not None:
        m.budget = m.budget0 = budget
    for ii, inst in enumerate(insts):  # the seed kernel
        m.live += 1
        m.live_prio[inst.prio] += 1
    for ii in range(len(insts)):
        m.next_wave(ii, 0)
    ctas = [CTA(m) for _ in range(grid)]
    idle_rounds = 0
    for _ in range(200000):
        progress = m.publish_one() if rng.random() < 0.5 else False
        order = list(range(grid))
        rng.shuffle(order)
        for c in order[: rng.randint(1, grid)]:
            progress |= ctas[c].step()
        if all(c.finished for c in ctas):
            break
        if progress:
            idle_rounds = 0
            continue
        # no step of the chosen CTAs moved: try every CTA and the producers once
        progress = m.publish_one() or any(c.step() for c in ctas)
        idle_rounds = 0 if progress else idle_rounds + 1
        assert idle_rounds < 3, "no CTA can make progress: the schedule is stuck"
    assert all(c.finished for c in ctas), "engine did not finish"
    for inst in insts:
        assert inst.retired
        assert [len(inst.seen.get(q, [])) for q in range(len(inst.waves) - 1)] == inst.waves[:-1]
    assert m.budget == m.budget0, "gang budget not returned"


@pytest.mark.parametrize("grid", [1, 2, 3, 5, 8, 16])
def test_schedule_model_finishes_every_wave(grid):
    for seed in range(12):
        run_model(seed * 31 + grid, grid, n2d=5 + seed % 4, n3d=seed % 5)


def test_schedule_model_many_volumes_small_grid():
    # more gang-eligible volumes than CTAs: the budget must keep claimers free
    for seed in range(20):
        run_model(1000 + seed, grid=4, n2d=1, n3d=8)


@pytest.mark.parametrize("grid", [2, 4, 6])
def test_schedule_model_smaller_budgets(grid):
    # the engine's budget is the whole grid; smaller ones only form fewer gangs
    for seed in range(15):
        run_model(3000 + 7 * seed + grid, grid=grid, n2d=2, n3d=6, budget=grid // 2)


def test_schedule_model_detects_the_dropped_eager_claim():
    """The model's own check: the design that took a fresh ticket while the
    tile was still being recorded (and waited for its item before publishing
    the tile's next wave) must get stuck in some interleavings."""
    stuck = 0
    for seed in range(40):
        try:
            run_model(2000 + seed, grid=2, n2d=2, n3d=0, eager_claim=True)
        except AssertionError as e:
            assert "stuck" in str(e) or "did not finish" in str(e)
            stuck += 1
    assert stuck > 0


def run_gang_vs_held_tickets(seed, held_first, grid=4):
    """A 2D instance whose waves (8 tiles on 4 CTAs) are deep enough for
    multiple claims, and a volume whose waves of 4 tiles form gangs as large
    as the whole grid, published at a random early step.  Returns False when
    the schedule gets stuck."""
    rng = random.Random(seed)
    a = Inst(rng, 2)
    a.waves = [8, 8, 8, 0]
    v = Inst(rng, 3)
    v.waves = [4] * 12 + [0]
    m = Model(rng, [a, v], grid)
    m.held_first = held_first
    for inst in m.insts:
        m.live += 1
        m.live_prio[inst.prio] += 1
    m.next_wave(0, 0)
    ctas = [CTA(m) for _ in range(grid)]
    publish_at = rng.randint(0, 30)
    published = False
    idle = 0
    for step in range(20000):
        if not published and step == publish_at:
            m.next_wave(1, 0)
            published = True
        progress = m.publish_one() if rng.random() < 0.5 else False
        order = list(range(grid))
        rng.shuffle(order)
        for c in order[: rng.randint(1, grid)]:
            progress |= ctas[c].step()
        if all(c.finished for c in ctas):
            return True
        if progress:
            idle = 0
            continue
        if not published:
            m.next_wave(1, 0)
            published = True
            continue
        progress = m.publish_one() or any(c.step() for c in ctas)
        idle = 0 if progress else idle + 1
        if idle >= 3:
            return False
    raise AssertionError("model did not finish within its step limit")


def test_gang_never_waits_on_a_ticket_holder():
    """A CTA holding bulk tickets used to be able to take a gang ticket first
    (ring 0 had priority over its held tickets); the 2D wave behind a held
    ticket then never finished while the gang waited for members.  The
    engine now consumes held tickets first: no interleaving gets stuck, and
    the model still finds the stall under the earlier rule."""
    assert all(run_gang_vs_held_tickets(s, held_first=True) for s in range(1500))
    assert not all(run_gang_vs_held_tickets(s, held_first=False) for s in range(1500))
