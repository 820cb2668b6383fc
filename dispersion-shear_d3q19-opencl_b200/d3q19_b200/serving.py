"""Served shear-rheology solves on one GPU: a request loop over the lattice
pool (continuous batching), and the one-at-a-time baseline it is measured
against.

A request is an independent shear cell: a cubic lattice with velocity walls
on z, periodic x and y, a viscosity law and a suspension of spheres.  It runs
until the domain-averaged shear stress (d3q19_mean_stress, FP64 on the
device) changes by less than `rel_tol` relative over `check_every` steps, or
until `max_steps`.

The server admits requests as they arrive, as long as a slot and HBM budget
are free; every member of the pool advances in the same batched launches, so
requests that arrive while others run overlap with them on the device, and a
finished request frees its memory for the queue.  With pre-emption on, a
request that does not fit may evict a long-running member (its checkpoint
goes to host memory, d3q19_pool_evict); the evicted member is re-admitted
(d3q19_pool_readmit) ahead of every request that arrived after its eviction
and continues bit for bit.  The reference has no counterpart (one lattice per
process); the physics of each request is the reference's.
"""
from __future__ import annotations

import dataclasses
import math
import threading
import time
from concurrent.futures import Future, ThreadPoolExecutor

import numpy as np

from . import D3Q19Error, HostState, Options, Pool, Simulation, keywords_text, parse_config

MODELS = ("newtonian", "power_law", "casson")


@dataclasses.dataclass
class ShearRequest:
    """One shear-rheology solve."""
    rid: int
    edge: tuple          # lattice size (incl. the 1-node buffer per face)
    phi: float           # sphere volume fraction
    model: str           # "newtonian" | "power_law" | "casson"
    wall_speed: float    # walls at +-wall_speed along x
    seed: int            # sphere placement seed
    arrival: float = 0.0  # seconds after the start of the sweep
    diameter: float = 8.0
    n_index: float = 0.6  # power-law index


def solve_keywords(req: ShearRequest) -> dict:
    """Input-file keywords (the reference's names, D3Q19-OpenCL.c:31-64, plus
    the placement and clamp keywords of this implementation) for a request."""
    N = tuple(int(v) for v in req.edge)
    r = req.diameter / 2.0
    # The wall repulsion (z_wall_particle_buffer) acts within r + 2 of a wall,
    # so markers stay off the wall planes (a marker that crosses one wraps to
    # the other wall, as in the reference); sphere centres start in the slab
    # beyond it, and phi is the volume fraction of that slab (random
    # sequential addition jams near 0.38).  The force smoothing wraps across
    # the periodic x/y seams (periodic_force_smoothing): with the reference's
    # smoothing a sphere on a seam loses part of its reaction on the fluid,
    # and dense suspensions build up velocity there until they diverge.
    zb = r + 2.0
    slab = (N[0] - 2) * (N[1] - 2) * max(N[2] - 2 - 2 * zb, 0.0)
    nsph = int(round(req.phi * slab / (4.0 / 3.0 * math.pi * r ** 3)))
    kw = dict(iterations=1_000_000, total_lattice_size=N, boundary_conditions_xyz=(0, 0, 1),
              velocity_bc_upper=(req.wall_speed, 0.0, 0.0), velocity_bc_lower=(-req.wall_speed, 0.0, 0.0),
              initial_f="constant", initial_vel=(0.0, 0.0, 0.0), domain_decomposition=(1, 1, 1),
              rebuild_neigh_list_freq=10, video_freq=10 ** 9, shear_stress_freq=10 ** 9, console_print_freq=10 ** 9,
              num_particles=nsph, periodic_force_smoothing=1)
    if nsph > 0:
        kw.update(particle_diameter=req.diameter, initial_particle_distribution=4, particle_seed=req.seed,
                  min_particle_gap=0.0, initial_particle_buffer=0.0, z_wall_particle_buffer=zb,
                  particle_collision_params=2.0)
    if req.model == "newtonian":
        kw.update(newtonian_tau=0.8, viscosity_model=1)
    elif req.model == "power_law":
        # Consistency k such that tau = 1 at the nominal shear rate 2U/H.
        rate = 2.0 * req.wall_speed / (N[2] - 2)
        k = (1.0 - 0.5) / 3.0 / rate ** (req.n_index - 1.0)
        kw.update(newtonian_tau=1.0, viscosity_model=2, viscosity_params=(k, req.n_index, 0.0, 0.0),
                  use_constant_viscosity=0, tau_min=0.55, tau_max=2.0)
    elif req.model == "casson":
        kw.update(newtonian_tau=0.8, viscosity_model=4, viscosity_params=(1e-4, (0.6 - 0.5) / 3.0, 0.0, 0.0),
                  use_constant_viscosity=0, casson_regularisation=1e-4, tau_max=2.0)
    else:
        raise ValueError(f"unknown model {req.model}")
    return kw


def host_state(req: ShearRequest, data_dir: str = ".") -> HostState:
    return HostState(parse_config(keywords_text(solve_keywords(req))), data_dir=data_dir)


def make_requests(n: int, rate: float, seed: int, edges=(32, 64), phi=(0.0, 0.3), models=MODELS,
                  wall_speed=0.02, diameter=8.0) -> list:
    """n requests with Poisson arrivals of mean rate `rate` per second, cubic
    edges uniform in [edges[0], edges[1]] (even), volume fractions uniform in
    phi and the viscosity law uniform over `models`; all from one seed."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        t += rng.exponential(1.0 / rate) if rate > 0 else 0.0
        e = int(rng.integers(edges[0] // 2, edges[1] // 2 + 1)) * 2
        out.append(ShearRequest(rid=i, edge=(e, e, e), phi=float(rng.uniform(*phi)),
                                model=str(models[int(rng.integers(len(models)))]), wall_speed=wall_speed,
                                seed=int(rng.integers(1, 2 ** 31 - 1)), arrival=t, diameter=diameter))
    return out


@dataclasses.dataclass
class SolveRecord:
    rid: int
    arrival: float
    start: float
    finish: float
    steps: int
    stress: float
    eff_viscosity: float
    converged: bool
    failed: bool = False  # the solve stopped on a device error (non-finite state)
    preempted: int = 0    # times the solve was evicted and re-admitted
    cancelled: bool = False  # stopped by Server.cancel

    @property
    def latency(self) -> float:
        return self.finish - self.arrival


class Convergence:
    """The stop rule: the mean shear stress changes by less than rel_tol
    (relative) between consecutive checks `check_every` steps apart."""

    def __init__(self, rel_tol: float = 1e-4):
        self.rel_tol = rel_tol
        self.last = None

    def update(self, stress: float) -> bool:
        prev, self.last = self.last, stress
        if prev is None:
            return False
        return abs(stress - prev) <= self.rel_tol * max(abs(stress), 1e-300)


def summary(records: list, wall: float) -> dict:
    lat = np.array([r.latency for r in records], np.float64)
    return {"solves": len(records), "wall_s": wall, "solves_per_s": len(records) / wall if wall > 0 else None,
            "p50_latency_s": float(np.percentile(lat, 50)) if len(lat) else None,
            "p99_latency_s": float(np.percentile(lat, 99)) if len(lat) else None,
            "converged": int(sum(r.converged for r in records)),
            "failed": int(sum(r.failed for r in records)),
            "preempted": int(sum(r.preempted for r in records)),
            "cancelled": int(sum(r.cancelled for r in records)),
            "steps": int(sum(r.steps for r in records))}


@dataclasses.dataclass
class _Member:
    req: ShearRequest
    start: float
    conv: Convergence
    base: int = 0        # pool step count at the (re)admission
    preempted: int = 0


class Server:
    """Continuous batching over a Pool: admit on arrival while slots and
    budget last, advance every member `check_every` steps at a time, retire
    the converged ones.  The host-side set-up of an arrived request (input
    parsing, sphere placement, initial state) runs on `builders` worker
    threads while the GPU works.

    preempt_after: None (off) or a step count.  When the request at the head
    of the queue does not fit, the member with the most steps since its
    (re)admission is evicted if that count is at least preempt_after, and
    again until the request fits or no member qualifies.  An evicted member
    is re-admitted before any request that arrived after its eviction.

    cancel(rid), from any thread, stops a request at the next chunk
    boundary: a queued one is never admitted, a running one is released, a
    parked one drops its checkpoint; its record has cancelled = True.

    solo_nodes: None (off) or an interior node count.  A request at least
    that large runs on a context of its own (the single-lattice kernels,
    faster per node than the batched ones, and a large lattice fills the GPU
    alone) instead of a pool slot, concurrently with the pool on its own
    stream, with the same stop rule; at most solo_slots of them at a time,
    within solo_budget bytes of device memory.  Admission stays in arrival
    order: a solo request that does not fit waits at the head of the queue.
    make_solo(hs) and solo_bytes(hs) create such a context and give its
    device bytes (by default a Simulation with the pool's storage and
    layout, and d3q19_context_bytes)."""

    def __init__(self, pool: Pool, check_every: int = 500, rel_tol: float = 1e-4, max_steps: int = 20000,
                 clock=time.perf_counter, sleep=time.sleep, builders: int = 4, preempt_after: int | None = None,
                 solo_nodes: int | None = None, solo_slots: int = 2, solo_budget: int = 32 << 30,
                 make_solo=None, solo_bytes=None):
        if check_every % pool.period:
            raise ValueError(f"check_every must be a multiple of the pool period {pool.period}")
        if preempt_after is not None and preempt_after <= 0:
            raise ValueError("preempt_after must be positive")
        if solo_nodes is not None and (solo_nodes <= 0 or solo_slots <= 0):
            raise ValueError("solo_nodes and solo_slots must be positive")
        self.solo_nodes = solo_nodes
        self.solo_slots = solo_slots
        self.solo_budget = solo_budget
        self.make_solo = make_solo or (lambda hs: Simulation.from_host_state(
            hs, device=pool.device, storage=pool.storage, inplace=pool.inplace))
        self.solo_bytes = solo_bytes or (lambda hs: _solo_context_bytes(hs, pool))
        self.pool = pool
        self.check_every = check_every
        self.rel_tol = rel_tol
        self.max_steps = max_steps
        self.clock = clock
        self.sleep = sleep
        self.builders = builders
        self.preempt_after = preempt_after
        self._lock = threading.Lock()
        self._cancel = set()

    def cancel(self, rid: int):
        """Asks to stop request rid (takes effect at the next chunk boundary)."""
        with self._lock:
            self._cancel.add(rid)

    def _cancelled(self):
        with self._lock:
            return set(self._cancel)

    def _stresses(self, active):
        """{slot: (stress, viscosity) or None for a failed member}."""
        out = {}
        if hasattr(self.pool, "mean_stress_all"):
            st, _, vi, code = self.pool.mean_stress_all(self.pool.max_slots)
            for slot in active:
                out[slot] = None if code[slot] != 0 else (float(st[slot]), float(vi[slot]))
            return out
        for slot in active:
            try:
                stress, _, visc = self.pool.member(slot).mean_stress()
                out[slot] = (stress, visc)
            except D3Q19Error:
                out[slot] = None
        return out

    def run(self, requests: list, build=host_state) -> tuple:
        """Serves the requests (arrival times relative to the call); returns
        (records in completion order, wall seconds)."""
        queue = sorted(requests, key=lambda r: r.arrival)
        t0 = self.clock()
        active = {}   # slot -> _Member
        joining = {}  # admitted while the pool was running: join the next chunk
        parked = []   # (queue index it waits for, _Member, checkpoint) in eviction order
        done = []
        ex = ThreadPoolExecutor(max_workers=self.builders) if self.builders > 0 else None
        built = {}  # rid -> Future or host state of an arrived request
        solo = {}   # rid -> _Solo: requests on contexts of their own
        qi = nb = 0

        def is_solo(req):
            return self.solo_nodes is not None and math.prod(e - 2 for e in req.edge) >= self.solo_nodes

        def solo_used():
            return sum(so.bytes for so in solo.values())

        def prepare():
            # Start the set-up of every request that has arrived.
            nonlocal nb
            now = self.clock() - t0
            while nb < len(queue) and queue[nb].arrival <= now:
                req = queue[nb]
                built[req.rid] = ex.submit(build, req) if ex else build(req)
                nb += 1

        def evict_one():
            # The member with the most steps since its (re)admission, if it
            # has run at least preempt_after of them.
            if self.preempt_after is None:
                return False
            best, run = None, -1
            for slot, m in active.items():
                n = self.pool.steps(slot) - m.base
                if n >= self.preempt_after and n > run:
                    best, run = slot, n
            if best is None:
                return False
            m = active.pop(best)
            m.preempted += 1
            parked.append((nb, m, self.pool.evict(best)))
            return True

        def make_room():
            # At a chunk boundary: while the request at the head of the queue
            # has arrived and does not fit, evict a long runner.  The request
            # is admitted while the next chunk runs.
            prepare()
            if self.preempt_after is None or qi >= nb or (parked and parked[0][0] <= qi):
                return
            req = queue[qi]
            if is_solo(req):  # not a pool member: evictions would not make room for it
                return
            hs = built[req.rid]
            if ex:
                hs = hs.result()
                built[req.rid] = _done_future(hs)
            while not self.pool.fits(hs) and evict_one():
                pass

        def admit_arrived():
            # Parked members that are due first, then arrivals in order; stop
            # at the first one that does not fit.
            nonlocal qi
            prepare()
            cancel_requested()
            while True:
                if parked and parked[0][0] <= qi:
                    _, m, ck = parked[0]
                    slot = self.pool.readmit(ck)
                    if slot is None:
                        return
                    parked.pop(0)
                    m.base = self.pool.steps(slot)
                    joining[slot] = m
                    continue
                if qi >= nb:
                    return
                req = queue[qi]
                hs = built[req.rid]
                if ex:
                    hs = hs.result()
                if is_solo(req):
                    nbytes = self.solo_bytes(hs)
                    if len(solo) >= self.solo_slots or solo_used() + nbytes > self.solo_budget:
                        built[req.rid] = hs if not ex else _done_future(hs)
                        if not solo and nbytes > self.solo_budget:
                            raise RuntimeError(f"request {req.rid} does not fit the solo budget")
                        return
                    del built[req.rid]
                    solo[req.rid] = _Solo(_Member(req, self.clock() - t0, Convergence(self.rel_tol)),
                                          self.make_solo(hs), nbytes)
                    qi += 1
                    continue
                slot = self.pool.admit(hs)
                if slot is None:
                    built[req.rid] = hs if not ex else _done_future(hs)
                    if not active and not joining and not solo:
                        raise RuntimeError(f"request {req.rid} does not fit an empty pool")
                    return
                del built[req.rid]
                joining[slot] = _Member(req, self.clock() - t0, Convergence(self.rel_tol), self.pool.steps(slot))
                qi += 1

        def cancel_requested():
            # Queued, parked and running requests asked to stop.
            nonlocal nb
            gone = self._cancelled()
            if not gone:
                return
            now = self.clock() - t0
            for members in (active, joining):
                for slot in [s for s, m in members.items() if m.req.rid in gone]:
                    m = members.pop(slot)
                    done.append(SolveRecord(m.req.rid, m.req.arrival, m.start, now, self.pool.steps(slot),
                                            float("nan"), float("nan"), False, False, m.preempted, True))
                    self.pool.release(slot)
            for rid in [r for r in solo if r in gone]:
                so = solo.pop(rid)
                done.append(SolveRecord(rid, so.m.req.arrival, so.m.start, now, so.t - 1, float("nan"),
                                        float("nan"), False, False, 0, True))
                so.sim.close()
            for entry in [e for e in parked if e[1].req.rid in gone]:
                parked.remove(entry)
                m = entry[1]
                done.append(SolveRecord(m.req.rid, m.req.arrival, m.start, now, 0, float("nan"), float("nan"), False,
                                        False, m.preempted, True))
            # Queued requests leave the queue; the ones behind them move up.
            dropped = [k for k in range(qi, len(queue)) if queue[k].rid in gone]
            if dropped:
                for k in dropped:
                    req = queue[k]
                    built.pop(req.rid, None)
                    done.append(SolveRecord(req.rid, req.arrival, now, now, 0, float("nan"), float("nan"), False,
                                            False, 0, True))
                nb -= sum(1 for k in dropped if k < nb)
                for j, (mark, m, ck) in enumerate(parked):
                    parked[j] = (mark - sum(1 for k in dropped if k < mark), m, ck)
                queue[:] = [r for k, r in enumerate(queue) if k < qi or r.rid not in gone]
            with self._lock:
                self._cancel -= gone

        try:
            while qi < len(queue) or active or joining or parked or solo:
                cancel_requested()
                if not (qi < len(queue) or active or joining or parked or solo):
                    break
                # Between chunks the GPU waits for the host, so requests are
                # admitted here only into an empty pool; otherwise they are
                # admitted while the next chunk runs.  Evictions need the
                # members' state at a chunk boundary: they happen here.
                if active or joining or solo:
                    make_room()
                else:
                    admit_arrived()
                active.update(joining)
                joining.clear()
                if not active and not solo:
                    if qi < len(queue):
                        self.sleep(max(0.0, queue[qi].arrival - (self.clock() - t0)))
                    continue
                # The chunk runs on the pool's stream (and the solo contexts'
                # chunks on theirs) while the host admits the requests that
                # arrived meanwhile (their set-up and first steps overlap the
                # chunk on the device); they join the next chunk.
                for so in solo.values():
                    so.sim.run(so.t, self.check_every)
                    so.t += self.check_every
                if active:
                    self.pool.advance(self.check_every)
                admit_arrived()
                for rid in list(solo):
                    so = solo[rid]
                    try:
                        stress, _, visc = so.sim.mean_stress()
                        failed = False
                    except D3Q19Error:
                        stress = visc = float("nan")
                        failed = True
                    ok = not failed and so.m.conv.update(stress)
                    if failed or ok or so.t - 1 >= self.max_steps:
                        done.append(SolveRecord(rid, so.m.req.arrival, so.m.start, self.clock() - t0, so.t - 1,
                                                stress, visc, ok, failed))
                        so.sim.close()
                        del solo[rid]
                if not active:
                    continue
                stresses = self._stresses(active)
                for slot in list(active):
                    m = active[slot]
                    req = m.req
                    steps = self.pool.steps(slot)
                    res = stresses[slot]
                    if res is None:
                        # A member whose state went non-finite retires as failed;
                        # the others are independent of it.
                        done.append(SolveRecord(req.rid, req.arrival, m.start, self.clock() - t0, steps,
                                                float("nan"), float("nan"), False, True, m.preempted))
                        self.pool.release(slot)
                        del active[slot]
                        continue
                    stress, visc = res
                    ok = m.conv.update(stress)
                    if ok or steps >= self.max_steps:
                        done.append(SolveRecord(req.rid, req.arrival, m.start, self.clock() - t0, steps, stress,
                                                visc, ok, False, m.preempted))
                        self.pool.release(slot)
                        del active[slot]
        finally:
            if ex:
                ex.shutdown(wait=True)
        return done, self.clock() - t0


@dataclasses.dataclass
class _Solo:
    m: _Member
    sim: object
    bytes: int
    t: int = 1  # next step


def _solo_context_bytes(hs, pool) -> int:
    from . import context_bytes

    opt = Options.from_buffer_copy(bytes(hs.options))
    opt.storage = pool.storage
    opt.inplace = pool.inplace
    return context_bytes(hs.cfg.ip, opt)


def _done_future(value):
    f = Future()
    f.set_result(value)
    return f


def one_at_a_time(requests: list, storage: int = 0, check_every: int = 500, rel_tol: float = 1e-4,
                  max_steps: int = 20000, device: int = 0, clock=time.perf_counter, sleep=time.sleep,
                  build=host_state) -> tuple:
    """The baseline: each request alone on the GPU, in arrival order (FP32 by
    default), with the same stop rule."""
    queue = sorted(requests, key=lambda r: r.arrival)
    t0 = clock()
    done = []
    for req in queue:
        wait = req.arrival - (clock() - t0)
        if wait > 0:
            sleep(wait)
        start = clock() - t0
        hs = build(req)
        sim = Simulation.from_host_state(hs, device=device, storage=storage)
        conv = Convergence(rel_tol)
        t, ok, failed = 1, False, False
        stress = visc = 0.0
        while t - 1 < max_steps:
            sim.run(t, check_every)
            t += check_every
            try:
                stress, _, visc = sim.mean_stress()
            except D3Q19Error:
                stress = visc = float("nan")
                failed = True
                break
            if conv.update(stress):
                ok = True
                break
        sim.close()
        done.append(SolveRecord(req.rid, req.arrival, start, clock() - t0, t - 1, stress, visc, ok, failed))
    return done, clock() - t0


__all__ = ["ShearRequest", "SolveRecord", "Convergence", "Server", "make_requests", "solve_keywords", "host_state",
           "one_at_a_time", "summary", "MODELS", "Options"]
