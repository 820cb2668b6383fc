"""The lattice pool (d3q19_pool_*, batched persistent kernels) on the GPU.

* A member's results are the same alone and in the mix: bit for bit, also
  when it joins while others are running (continuous batching).
* A member matches the same solve run on its own context (to the fast
  path's tolerance: the pool's kernel picks the viscosity law at run time).
* Admission respects the HBM budget; release frees it.
* The serving loop drives requests to completion.
"""
import numpy as np
import pytest

import d3q19_b200 as d3
from d3q19_b200 import serving as sv
from gpu_helpers import REL_TOL, rel_l2

pytestmark = pytest.mark.gpu

REQS = [
    sv.ShearRequest(rid=0, edge=(34, 34, 34), phi=0.2, model="newtonian", wall_speed=0.02, seed=3),
    sv.ShearRequest(rid=1, edge=(42, 42, 42), phi=0.25, model="power_law", wall_speed=0.03, seed=4),
    sv.ShearRequest(rid=2, edge=(36, 36, 36), phi=0.0, model="casson", wall_speed=0.02, seed=5),
    sv.ShearRequest(rid=3, edge=(32, 40, 36), phi=0.1, model="casson", wall_speed=0.01, seed=6),
]


def state(pool, slot):
    m = pool.member(slot)
    out = {"u": m.read_u(), "tau": m.read_tau(), "stress": np.array(m.mean_stress())}
    if m.np > 0:
        out["kin"] = m.read_parkin()
        out["pff"] = m.read_parfluidforce()
    return out


def bits_equal(a, b):
    for k in a:
        x, y = np.ascontiguousarray(a[k]), np.ascontiguousarray(b[k])
        assert x.shape == y.shape and np.array_equal(x.view(np.uint8), y.view(np.uint8)), k


def alone(req, storage, schedule, inplace=False):
    pool = d3.Pool(storage=storage, max_slots=4, inplace=inplace)
    s = pool.admit(sv.host_state(req))
    for n in schedule:
        pool.advance(n)
    out = state(pool, s)
    pool.close()
    return out


@pytest.mark.parametrize("storage", [0, 1])
def test_members_identical_alone_and_in_the_mix(storage):
    pool = d3.Pool(storage=storage, max_slots=8)
    # Members 0 and 1 first; 2 and 3 join after 100 steps (reverse order, so
    # their slots differ from the runs alone).
    s0 = pool.admit(sv.host_state(REQS[0]))
    s1 = pool.admit(sv.host_state(REQS[1]))
    pool.advance(100)
    s3 = pool.admit(sv.host_state(REQS[3]))
    s2 = pool.admit(sv.host_state(REQS[2]))
    pool.advance(200)
    mixed = {0: state(pool, s0), 1: state(pool, s1), 2: state(pool, s2), 3: state(pool, s3)}
    assert pool.steps(s0) == pool.period + 300 and pool.steps(s2) == pool.period + 200
    pool.close()
    bits_equal(mixed[0], alone(REQS[0], storage, [100, 200]))
    bits_equal(mixed[1], alone(REQS[1], storage, [300]))
    bits_equal(mixed[2], alone(REQS[2], storage, [200]))
    bits_equal(mixed[3], alone(REQS[3], storage, [100, 100]))


def test_release_in_flight_and_memory_reuse():
    # A release returns without waiting for the chunk in flight (the member's
    # memory is freed in the pool stream's order); a member admitted right
    # after it may reuse that memory.  Neither the member that stays nor the
    # newcomer sees the difference.
    pool = d3.Pool(storage=0, max_slots=4)
    s0 = pool.admit(sv.host_state(REQS[0]))
    s1 = pool.admit(sv.host_state(REQS[1]))
    pool.advance(100)
    pool.release(s1)  # the 100-step chunk is still queued or running
    s2 = pool.admit(sv.host_state(REQS[2]))
    pool.advance(100)
    pool.release(s0)
    s3 = pool.admit(sv.host_state(REQS[3]))
    pool.advance(100)
    got = {0: None, 2: state(pool, s2), 3: state(pool, s3)}
    assert pool.steps(s2) == pool.period + 200 and pool.steps(s3) == pool.period + 100
    pool.close()
    bits_equal(got[2], alone(REQS[2], 0, [100, 100]))
    bits_equal(got[3], alone(REQS[3], 0, [100]))


@pytest.mark.parametrize("rid", [0, 1, 2])
def test_member_matches_its_own_context(rid):
    req = REQS[rid]
    pool = d3.Pool(storage=0, max_slots=2)
    s = pool.admit(sv.host_state(req))
    pool.advance(200)
    got = state(pool, s)
    n = pool.steps(s)
    pool.close()
    sim = d3.Simulation.from_host_state(sv.host_state(req))
    sim.run(1, n)
    # The pool's kernel chooses the viscosity law at run time, the context's
    # is compiled for it: the same arithmetic up to contraction, so the fast
    # path's tolerance -- except in a Casson plug, whose relaxation rate is the
    # reciprocal of a rounding-level strain rate (the reference itself moves
    # by 3.4e-4 in u under contraction, tests/golden/rounding_spread.json).
    tol = 1e-3 if req.model == "casson" else REL_TOL
    assert rel_l2(got["u"], sim.read_u()) <= tol
    if sim.np > 0:
        k, kr = got["kin"].reshape(-1, 4), sim.read_parkin().reshape(-1, 4)
        assert rel_l2(k[:sim.np, :3], kr[:sim.np, :3]) <= REL_TOL
    st = np.array(sim.mean_stress())
    assert np.allclose(got["stress"], st, rtol=1e-4, atol=1e-12)
    sim.close()


def test_admission_within_budget_and_release():
    a, b = sv.host_state(REQS[0]), sv.host_state(REQS[1])
    need_a = d3.context_bytes(a.cfg.ip, a.options)
    probe = d3.Pool(storage=0, max_slots=4)
    base, _, _ = probe.usage()  # the pool's own argument arrays (4 slots)
    probe.close()
    pool = d3.Pool(storage=0, max_slots=4, hbm_budget=base + need_a + 1024)
    sa = pool.admit(a)
    assert sa is not None
    assert pool.admit(b) is None  # over budget: EBUSY, nothing allocated
    used, budget, n = pool.usage()
    assert n == 1 and used == base + need_a and budget == base + need_a + 1024
    pool.advance(20)
    pool.release(sa)
    assert pool.usage()[2] == 0
    pool.close()
    pool = d3.Pool(storage=0, max_slots=4, hbm_budget=base + d3.context_bytes(b.cfg.ip, b.options))
    assert pool.admit(b) is not None
    pool.close()


def test_server_serves_a_burst():
    reqs = [sv.ShearRequest(rid=i, edge=(32, 32, 32), phi=0.1, model=sv.MODELS[i % 3], wall_speed=0.02,
                            seed=10 + i, arrival=0.0) for i in range(6)]
    pool = d3.Pool(storage=1, max_slots=8)
    recs, wall = sv.Server(pool, check_every=100, rel_tol=1e-4, max_steps=600).run(reqs)
    assert sorted(r.rid for r in recs) == list(range(6))
    assert pool.usage()[2] == 0
    assert all(r.steps <= 600 + pool.period and np.isfinite(r.stress) for r in recs)
    pool.close()


def test_batched_stress_matches_per_member():
    pool = d3.Pool(storage=1, max_slots=6)
    slots = [pool.admit(sv.host_state(r)) for r in REQS]
    pool.advance(100)
    st, ra, vi, code = pool.mean_stress_all(6)
    for s in slots:
        one = pool.member(s).mean_stress()
        assert code[s] == 0
        assert (st[s], ra[s], vi[s]) == one
    free = [k for k in range(6) if k not in slots]
    assert all(code[k] == -1 and np.isnan(st[k]) for k in free)
    pool.close()


def test_server_preemption_changes_no_result():
    # A pool that holds two of the six solves at a time, served in arrival
    # order and with pre-emption: evicted solves continue from their
    # checkpoints, so every solve ends with the same steps and bit-identical
    # stress and viscosity either way.
    reqs = [sv.ShearRequest(rid=i, edge=(32 + 2 * (i % 3),) * 3, phi=0.1, model=sv.MODELS[i % 3], wall_speed=0.02,
                            seed=20 + i, arrival=0.0) for i in range(6)]
    need = 0
    for r in reqs:
        h = sv.host_state(r)
        opt = d3.Options.from_buffer_copy(bytes(h.options))
        opt.storage = 1
        need = max(need, d3.context_bytes(h.cfg.ip, opt))
    probe = d3.Pool(storage=1, max_slots=6)
    base, _, _ = probe.usage()
    probe.close()
    out = {}
    for pre in (None, 300):
        pool = d3.Pool(storage=1, max_slots=6, hbm_budget=base + 2 * need + need // 2)
        recs, _ = sv.Server(pool, check_every=100, rel_tol=1e-12, max_steps=1500, builders=0,
                            preempt_after=pre).run(reqs)
        assert pool.usage()[2] == 0
        pool.close()
        out[pre] = {r.rid: r for r in recs}
    assert sum(r.preempted for r in out[300].values()) > 0
    for i in range(6):
        a, b = out[None][i], out[300][i]
        assert a.steps == b.steps and a.stress == b.stress and a.eff_viscosity == b.eff_viscosity, i


def test_pool_driven_from_several_threads():
    # Every pool call holds the pool's lock: members admitted from four
    # threads at once, and a member admitted while another thread advances
    # the pool, end bit for bit like the same solves alone.
    import threading

    pool = d3.Pool(storage=1, max_slots=8)
    states = [sv.host_state(r) for r in REQS]
    slots = [None] * 4
    errs = []

    def admit(k):
        try:
            slots[k] = pool.admit(states[k])
        except Exception as e:  # noqa: BLE001 - reported by the assert below
            errs.append(e)

    th = [threading.Thread(target=admit, args=(k,)) for k in range(3)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not errs and None not in slots[:3]

    def drive():
        try:
            for _ in range(5):
                pool.advance(20)
        except Exception as e:  # noqa: BLE001
            errs.append(e)

    t = threading.Thread(target=drive)
    t.start()
    admit(3)  # while the chunks run
    t.join()
    pool.advance(20)
    assert not errs and slots[3] is not None
    got = {k: (state(pool, slots[k]), pool.steps(slots[k]) - pool.period) for k in range(4)}
    pool.close()
    assert got[0][1] == 120
    for k in range(4):
        bits_equal(got[k][0], alone(REQS[k], 1, [got[k][1]]))


def test_poll_reports_the_chunk_without_waiting():
    import time

    pool = d3.Pool(storage=1, max_slots=2)
    assert pool.poll()  # nothing queued yet
    pool.admit(sv.host_state(REQS[1]))
    pool.advance(2000)
    t0 = time.perf_counter()
    while not pool.poll():
        assert time.perf_counter() - t0 < 60.0
        time.sleep(0.001)
    pool.synchronize()
    assert pool.poll()
    pool.close()


def test_non_finite_member_is_reported_and_isolated():
    # A NaN planted (from the host) in one member's populations: the device
    # error word of that member reports it (ENUMERIC) while the other member
    # runs on bit for bit as alone, and the GPU stays usable.
    pool = d3.Pool(storage=0, max_slots=4)
    sa = pool.admit(sv.host_state(REQS[0]))
    sb = pool.admit(sv.host_state(REQS[2]))
    m = pool.member(sb)
    f = m.read_f()
    N = m.ip.LatticeSize
    centre = N[0] // 2 + N[0] * (N[1] // 2 + N[1] * (N[2] // 2))  # an interior node
    f[5 * m.nc + centre] = np.nan
    m.write_lattice(f, m.read_u(), m.read_tau())
    pool.advance(20)
    st, _, _, code = pool.mean_stress_all(4)
    assert d3.STATUS[int(code[sb])] == "ENUMERIC" and code[sa] == 0 and np.isfinite(st[sa])
    pool.release(sb)
    pool.advance(20)
    got = state(pool, sa)
    pool.close()
    bits_equal(got, alone(REQS[0], 0, [40]))


def test_non_finite_state_is_reported_by_a_context():
    hs = sv.host_state(REQS[2])
    sim = d3.Simulation.from_host_state(hs)
    f = np.array(hs.f, np.float32, copy=True).reshape(-1)
    N = sim.ip.LatticeSize
    f[3 * sim.nc + N[0] // 2 + N[0] * (N[1] // 2 + N[1] * (N[2] // 2))] = np.inf  # an interior node
    sim.write_lattice(f, hs.u, hs.tau)
    sim.run(1, 4)
    with pytest.raises(d3.D3Q19Error, match="ENUMERIC"):
        sim.synchronize()
    with pytest.raises(d3.D3Q19Error, match="ENUMERIC"):  # sticky: reported by every later call
        sim.read_u()
    sim.close()
    ok = d3.Simulation.from_host_state(hs)
    ok.run(1, 4)
    ok.synchronize()
    assert np.isfinite(ok.read_u()).all()
    ok.close()


def test_server_cancels_queued_and_running_requests():
    reqs = [sv.ShearRequest(rid=i, edge=(32, 32, 32), phi=0.1, model=sv.MODELS[i % 3], wall_speed=0.02,
                            seed=30 + i, arrival=0.0) for i in range(4)]
    pool = d3.Pool(storage=0, max_slots=8)
    srv = sv.Server(pool, check_every=100, rel_tol=1e-12, max_steps=1000, builders=0)
    srv.cancel(3)
    advance, chunks = pool.advance, []

    def advance_then_cancel(n):  # as another thread would, while chunk 2 runs
        advance(n)
        chunks.append(n)
        if len(chunks) == 2:
            srv.cancel(1)

    pool.advance = advance_then_cancel
    recs, _ = srv.run(reqs)
    by = {r.rid: r for r in recs}
    assert by[3].cancelled and by[3].steps == 0
    assert by[1].cancelled and by[1].steps < 1000
    assert not by[0].cancelled and by[0].steps >= 1000 and np.isfinite(by[0].stress)
    assert pool.usage()[2] == 0
    pool.close()



@pytest.mark.parametrize("storage", [0, 1])
def test_inplace_pool_matches_two_buffer_pool(storage):
    # Members with one distribution buffer (in place): identical alone and in
    # the mix with late joins, and bit for bit the two-buffer members.
    pool = d3.Pool(storage=storage, max_slots=8, inplace=True)
    s0 = pool.admit(sv.host_state(REQS[0]))
    s1 = pool.admit(sv.host_state(REQS[1]))
    pool.advance(100)
    s3 = pool.admit(sv.host_state(REQS[3]))
    pool.advance(60)
    got = {0: state(pool, s0), 1: state(pool, s1), 3: state(pool, s3)}
    # A two-buffer member does not join an in-place pool.
    with pytest.raises(d3.D3Q19Error, match="EINVAL"):
        pool.admit(sv.host_state(REQS[2]), inplace=0)
    pool.close()
    bits_equal(got[0], alone(REQS[0], storage, [100, 60]))
    bits_equal(got[0], alone(REQS[0], storage, [160], inplace=True))
    bits_equal(got[1], alone(REQS[1], storage, [160]))
    bits_equal(got[3], alone(REQS[3], storage, [60]))


def test_inplace_pool_evict_and_readmit():
    pool = d3.Pool(storage=0, max_slots=4, inplace=True)
    sa = pool.admit(sv.host_state(REQS[0]))
    sb = pool.admit(sv.host_state(REQS[1]))
    pool.advance(40)
    ev = pool.evict(sa)
    pool.advance(20)
    sa = pool.readmit(ev)
    pool.advance(40)
    got = state(pool, sa)
    pool.close()
    bits_equal(got, alone(REQS[0], 0, [80]))
