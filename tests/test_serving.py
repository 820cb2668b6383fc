"""Host logic of the served sweep (no GPU): request generation, the stop
rule, and the continuous-batching loop driven against a fake pool that
counts steps and models the HBM budget."""
import numpy as np
import pytest

import d3q19_b200 as d3
from d3q19_b200 import serving as sv


def test_requests_are_seeded_and_poisson():
    a = sv.make_requests(400, 50.0, 11)
    b = sv.make_requests(400, 50.0, 11)
    assert [(r.edge, r.phi, r.model, r.seed, r.arrival) for r in a] == \
        [(r.edge, r.phi, r.model, r.seed, r.arrival) for r in b]
    gaps = np.diff([0.0] + [r.arrival for r in a])
    assert gaps.mean() == pytest.approx(1 / 50.0, rel=0.15)
    assert all(32 <= r.edge[0] <= 64 and r.edge[0] % 2 == 0 for r in a)
    assert {r.model for r in a} == set(sv.MODELS)
    assert all(0.0 <= r.phi <= 0.3 for r in a)


@pytest.mark.parametrize("model", sv.MODELS)
def test_request_builds_reference_initial_state(model):
    req = sv.ShearRequest(rid=0, edge=(34, 34, 34), phi=0.2, model=model, wall_speed=0.02, seed=5)
    hs = sv.host_state(req)
    ip = hs.cfg.ip
    assert tuple(ip.LatticeSize) == (34, 34, 34) and tuple(ip.BoundaryConds) == (0, 0, 1)
    assert ip.NumParticles > 0
    assert ip.ViscosityModel == {"newtonian": 1, "power_law": 2, "casson": 4}[model]
    assert hs.options.variable_viscosity == (model != "newtonian")
    z = hs.parKin.reshape(-1, 4)[:ip.NumParticles, 2]
    assert np.all(z >= 6.0) and np.all(z <= 32.0 - 6.0)  # radius + 2 off the walls
    assert hs.cfg.fp.ParticleZBuffer == 6.0


def test_stop_rule():
    c = sv.Convergence(1e-4)
    assert not c.update(1.0)
    assert not c.update(1.001)
    assert c.update(1.00105)


class FakeMember:
    def __init__(self, pool, slot, target):
        self.pool, self.slot, self.target = pool, slot, target

    def mean_stress(self):
        s = self.pool.steps_done[self.slot]
        # Relaxes towards the target: converges after a request-dependent time.
        return self.target * (1.0 - np.exp(-s / self.pool.tconst.get(self.slot, 1000.0))), 0.0, 0.0


class FakePool:
    period = 10

    def __init__(self, budget):
        self.budget, self.used = budget, 0
        self.steps_done, self.size, self.target, self.tconst, self.rid = {}, {}, {}, {}, {}
        self.admitted, self.max_members, self.next = [], 0, 0
        self.evicted, self.readmitted = [], []
        self.events, self.now = [], lambda: 0.0  # (kind, rid, time) in call order

    def admit(self, hs, steps=None):
        b = hs["bytes"]
        if self.used + b > self.budget:
            return None
        s = self.next
        self.next += 1
        self.used += b
        self.size[s], self.target[s] = b, hs["target"]
        self.steps_done[s] = self.period if steps is None else steps
        self.tconst[s] = hs.get("tconst", 1000.0)
        self.rid[s] = hs["rid"]
        if steps is None:
            self.admitted.append(hs["rid"])
            self.events.append(("admit", hs["rid"], self.now()))
        self.max_members = max(self.max_members, len(self.size))
        return s

    def fits(self, hs):
        return self.used + hs["bytes"] <= self.budget

    # Checkpoints hold the member's state: its step count and parameters.
    def evict(self, s):
        assert self.steps_done[s] % self.period == 0
        ck = ({"bytes": self.size[s], "rid": self.rid[s], "target": self.target[s], "tconst": self.tconst[s]},
              self.steps_done[s])
        self.evicted.append(ck[0]["rid"])
        self.events.append(("evict", ck[0]["rid"], self.now()))
        self.release(s)
        return ck

    def readmit(self, ck):
        slot = self.admit(ck[0], steps=ck[1])
        if slot is not None:
            self.readmitted.append(ck[0]["rid"])
            self.events.append(("readmit", ck[0]["rid"], self.now()))
        return slot


    def advance(self, n):
        for s in self.size:
            self.steps_done[s] += n

    def member(self, s):
        return FakeMember(self, s, self.target[s])

    def steps(self, s):
        return self.steps_done[s]

    def release(self, s):
        self.used -= self.size.pop(s)



def test_server_admits_in_order_within_budget_and_retires():
    # A burst: all twelve are waiting from the start.
    reqs = [sv.ShearRequest(rid=i, edge=(32, 32, 32), phi=0.0, model="newtonian", wall_speed=0.02, seed=1,
                            arrival=1e-6 * i) for i in range(12)]
    pool = FakePool(budget=4 * 10)
    clock = {"t": 0.0}

    def now():
        clock["t"] += 1e-4
        return clock["t"]

    srv = sv.Server(pool, check_every=500, rel_tol=1e-4, max_steps=30000, clock=now,
                    sleep=lambda dt: clock.__setitem__("t", clock["t"] + dt))
    build = lambda r: {"bytes": 10, "rid": r.rid, "target": 1.0 + r.rid}
    recs, wall = srv.run(reqs, build=build)
    assert sorted(r.rid for r in recs) == list(range(12))
    assert pool.admitted == list(range(12))  # arrival order
    assert pool.max_members == 4             # the budget holds 4 at a time
    assert pool.used == 0
    assert all(r.converged for r in recs)
    assert all(r.finish >= r.start >= r.arrival for r in recs)
    s = sv.summary(recs, wall)
    assert s["solves"] == 12 and s["p99_latency_s"] >= s["p50_latency_s"] > 0


def test_server_rejects_check_interval_off_the_period():
    with pytest.raises(ValueError):
        sv.Server(FakePool(10), check_every=505)


def test_context_bytes_counts_the_distributions():
    cfg = d3.parse_config("total_lattice_size 64 64 64\nboundary_conditions_xyz 0 0 1\nnum_particles 0\n")
    b32 = d3.context_bytes(cfg.ip, d3.Options())
    o = d3.Options()
    o.storage = 1
    b16 = d3.context_bytes(cfg.ip, o)
    nc = 64 ** 3
    assert b32 >= 2 * 19 * 4 * nc + 16 * nc and b32 - b16 == pytest.approx(2 * 19 * 2 * nc, rel=1e-3)


class FailingMember(FakeMember):
    def mean_stress(self):
        if self.pool.steps_done[self.slot] > 1000:
            raise d3.D3Q19Error("mean_stress: ENUMERIC: non-finite")
        return super().mean_stress()


def test_server_retires_a_failed_member_and_goes_on():
    reqs = [sv.ShearRequest(rid=i, edge=(32, 32, 32), phi=0.0, model="newtonian", wall_speed=0.02, seed=1,
                            arrival=0.0) for i in range(3)]
    pool = FakePool(budget=100)
    orig = pool.member
    pool.member = lambda s: FailingMember(pool, s, pool.target[s]) if s == 1 else orig(s)
    recs, wall = sv.Server(pool, check_every=500, max_steps=30000, clock=lambda: 0.0, sleep=lambda dt: None).run(
        reqs, build=lambda r: {"bytes": 10, "rid": r.rid, "target": 1.0})
    by = {r.rid: r for r in recs}
    assert by[1].failed and not by[1].converged and by[0].converged and by[2].converged
    assert sv.summary(recs, 1.0)["failed"] == 1 and pool.used == 0


def serve_long_then_short(preempt_after):
    # One slot's worth of budget; a long solve arrives first, three short ones
    # just after it.
    reqs = [sv.ShearRequest(rid=i, edge=(32, 32, 32), phi=0.0, model="newtonian", wall_speed=0.02, seed=1,
                            arrival=1e-3 * i) for i in range(4)]
    pool = FakePool(budget=10)
    clock = {"t": 0.0}

    def now():
        clock["t"] += 1e-4
        return clock["t"]

    build = lambda r: {"bytes": 10, "rid": r.rid, "target": 1.0, "tconst": 4000.0 if r.rid == 0 else 200.0}
    srv = sv.Server(pool, check_every=500, rel_tol=1e-4, max_steps=60000, clock=now,
                    sleep=lambda dt: clock.__setitem__("t", clock["t"] + dt), builders=0,
                    preempt_after=preempt_after)
    recs, wall = srv.run(reqs, build=build)
    return {r.rid: r for r in recs}, pool


def test_preemption_lets_short_solves_past_a_long_one():
    plain, pool0 = serve_long_then_short(None)
    pre, pool1 = serve_long_then_short(3000)
    assert pool0.evicted == [] and [r.rid for r in sorted(plain.values(), key=lambda r: r.finish)] == [0, 1, 2, 3]
    # With pre-emption the long solve is evicted (checkpointed) once the short
    # ones wait, and finishes last.
    assert pool1.evicted and set(pool1.evicted) == {0} and pool1.readmitted == pool1.evicted
    assert max(pre.values(), key=lambda r: r.finish).rid == 0 and pre[0].preempted == len(pool1.evicted)
    # Every solve takes the same steps either way (it continues from its
    # checkpoint), the short ones finish earlier, and the pool ends empty.
    assert all(pre[i].steps == plain[i].steps and pre[i].converged for i in range(4))
    assert all(pre[i].finish < plain[i].finish for i in (1, 2, 3))
    assert pool1.used == 0 and sv.summary(list(pre.values()), 1.0)["preempted"] == pre[0].preempted


def test_preempted_member_is_not_starved():
    # Arrivals keep coming: an evicted member is re-admitted before every
    # request that arrived after its eviction.
    reqs = [sv.ShearRequest(rid=i, edge=(32, 32, 32), phi=0.0, model="newtonian", wall_speed=0.02, seed=1,
                            arrival=0.0 if i == 0 else 0.004 * i) for i in range(12)]
    arrival = {r.rid: r.arrival for r in reqs}
    pool = FakePool(budget=20)
    clock = {"t": 0.0}

    def now():
        clock["t"] += 1e-3
        return clock["t"]

    pool.now = lambda: clock["t"]
    build = lambda r: {"bytes": 10, "rid": r.rid, "target": 1.0, "tconst": 3000.0 if r.rid % 4 == 0 else 400.0}
    recs, _ = sv.Server(pool, check_every=500, max_steps=60000, clock=now,
                        sleep=lambda dt: clock.__setitem__("t", clock["t"] + dt), builders=0,
                        preempt_after=1000).run(reqs, build=build)
    assert sorted(r.rid for r in recs) == list(range(12)) and all(r.converged for r in recs)
    assert pool.evicted and sorted(pool.readmitted) == sorted(pool.evicted) and pool.used == 0
    ev = pool.events
    for i, (kind, rid, te) in enumerate(ev):
        if kind != "evict":
            continue
        j = next(k for k in range(i + 1, len(ev)) if ev[k][:2] == ("readmit", rid))
        # Admitted while it waited: only requests that had arrived by its eviction.
        assert all(arrival[r] <= te for kd, r, _ in ev[i + 1:j] if kd == "admit")


def test_preempt_after_must_be_positive():
    with pytest.raises(ValueError):
        sv.Server(FakePool(10), check_every=500, preempt_after=0)


def test_cancel_queued_running_and_parked():
    reqs = [sv.ShearRequest(rid=i, edge=(32, 32, 32), phi=0.0, model="newtonian", wall_speed=0.02, seed=1,
                            arrival=1e-3 * i) for i in range(5)]
    clock = {"t": 0.0}

    def now():
        clock["t"] += 1e-4
        return clock["t"]

    class HookPool(FakePool):
        # Calls the hook after every advance, as another thread would.
        hook = None

        def advance(self, n):
            super().advance(n)
            if self.hook:
                self.hook(self)

    pool = HookPool(budget=20)
    srv = sv.Server(pool, check_every=500, rel_tol=1e-4, max_steps=60000, clock=now,
                    sleep=lambda dt: clock.__setitem__("t", clock["t"] + dt), builders=0, preempt_after=1000)
    build = lambda r: {"bytes": 10, "rid": r.rid, "target": 1.0, "tconst": 3000.0 if r.rid in (0, 1) else 300.0}
    srv.cancel(4)  # queued: never admitted

    def hook(p):
        members = {p.rid[s]: s for s in p.size}
        if 0 in members and p.steps_done[members[0]] >= 2000:
            srv.cancel(0)  # running
        if 1 in p.evicted and 1 not in members and 1 not in p.readmitted:
            srv.cancel(1)  # parked after its eviction

    pool.hook = hook
    recs, _ = srv.run(reqs, build=build)
    by = {r.rid: r for r in recs}
    assert sorted(by) == [0, 1, 2, 3, 4]
    assert by[4].cancelled and by[4].steps == 0 and 4 not in pool.admitted
    assert by[0].cancelled and 2000 <= by[0].steps < 60000
    assert all(by[k].converged and not by[k].cancelled for k in (2, 3))
    assert pool.used == 0 and sv.summary(recs, 1.0)["cancelled"] == sum(r.cancelled for r in recs)
    assert 1 in pool.evicted and by[1].cancelled and 1 not in pool.readmitted


class FakeSolo:
    live = 0
    peak = 0

    def __init__(self, hs):
        self.hs, self.steps = hs, 0
        FakeSolo.live += 1
        FakeSolo.peak = max(FakeSolo.peak, FakeSolo.live)

    def run(self, t0, n):
        assert t0 == self.steps + 1
        self.steps += n

    def mean_stress(self):
        return self.hs["target"] * (1.0 - np.exp(-self.steps / 1000.0)), 0.0, 0.0

    def close(self):
        FakeSolo.live -= 1


def test_large_requests_run_on_contexts_of_their_own():
    """solo_nodes: requests at least that large bypass the pool and run on
    their own contexts (at most solo_slots at a time, within solo_budget),
    in arrival order, with the same stop rule; the small ones share the
    pool meanwhile."""
    edges = [32, 160, 40, 150, 36, 140, 34, 130]
    reqs = [sv.ShearRequest(rid=i, edge=(e, e, e), phi=0.0, model="newtonian", wall_speed=0.02, seed=1,
                            arrival=0.0) for i, e in enumerate(edges)]
    pool = FakePool(budget=100)
    FakeSolo.live = FakeSolo.peak = 0
    build = lambda r: {"bytes": 10, "rid": r.rid, "target": 1.0 + r.rid, "edge": r.edge[0]}
    srv = sv.Server(pool, check_every=500, rel_tol=1e-4, max_steps=30000, clock=lambda: 0.0,
                    sleep=lambda dt: None, solo_nodes=100 ** 3, solo_slots=2, solo_budget=25,
                    make_solo=FakeSolo, solo_bytes=lambda hs: 10)
    recs, _ = srv.run(reqs, build=build)
    assert sorted(r.rid for r in recs) == list(range(8))
    assert pool.admitted == [0, 2, 4, 6]          # the small ones only
    assert FakeSolo.peak == 2 and FakeSolo.live == 0
    assert all(r.converged and r.steps % 500 == 0 for r in recs if r.rid % 2)
    assert all(r.converged for r in recs)
    with pytest.raises(ValueError):
        sv.Server(pool, solo_nodes=0)
