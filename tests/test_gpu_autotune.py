"""The pool's grid autotuner (d3q19_pool_autotune) on the GPU: it picks the
particle and contact grids (the fluid pass runs one CTA per tile).

* Advances of at least 100 steps time the candidates of the pool's work
  class one by one; once all have run, the fastest is kept and used.
* The tuning changes no result: the members end bit for bit where a pool
  with a fixed grid leaves them.
* Shorter advances are not timed; a long advance times one candidate per
  100-step segment.
* The table exported by one process seeds another: an imported class is
  settled at once.
"""
import math

import numpy as np
import pytest

import d3q19_b200 as d3
from d3q19_b200 import serving as sv
from test_gpu_pool import REQS, bits_equal, state

pytestmark = pytest.mark.gpu


def pool_with(reqs, autotune, storage=1):
    pool = d3.Pool(storage=storage, max_slots=4, autotune=autotune)
    slots = [pool.admit(sv.host_state(r)) for r in reqs]
    return pool, slots


def test_tuner_settles_on_the_fastest_and_changes_no_result():
    d3.tune_clear()
    pool, slots = pool_with(REQS[:2], True)
    st = pool.tune_state()
    pool.advance(20)  # too short to be timed
    st = pool.tune_state()
    assert st["tried"] == 0 and not st["settled"] and st["candidates"] == 3
    n = 20
    while not pool.tune_state()["settled"]:
        pool.advance(100)
        n += 100
        assert n <= 20 + 100 * 4
    trials = pool.tune_trials()
    assert len(trials) == 3 and all(f == 0 and t is not None and t > 0 for f, _, t in trials)
    best = min(trials, key=lambda x: x[2])
    pool.advance(100)  # runs with the choice
    n += 100
    st = pool.tune_state()
    assert (st["fluid_ctas_per_sm"], st["particle_ctas_per_sm"]) == best[:2]
    tuned = [state(pool, s) for s in slots]
    pool.close()
    print("trials (fluid, particle CTAs/SM, ns per tile step):", trials)
    fixed, slots = pool_with(REQS[:2], False)
    fixed.advance(20)
    fixed.advance(n - 20)
    for s, t in zip(slots, tuned):
        bits_equal(t, state(fixed, s))
    fixed.close()
    assert any(line.split("\t")[2] == "1" for line in d3.tune_export().splitlines())


def test_imported_class_is_settled_at_once():
    d3.tune_clear()
    pool, _ = pool_with(REQS[:1], True, storage=0)
    while not pool.tune_state()["settled"]:
        pool.advance(100)
    choice = pool.tune_state()
    text = d3.tune_export()
    pool.close()
    d3.tune_clear()
    d3.tune_import(text)
    pool, _ = pool_with(REQS[:1], True, storage=0)
    pool.advance(100)
    st = pool.tune_state()
    assert st["settled"] and st["tried"] == 1 and st["candidates"] == 1
    assert (st["fluid_ctas_per_sm"], st["particle_ctas_per_sm"]) == \
        (choice["fluid_ctas_per_sm"], choice["particle_ctas_per_sm"])
    pool.close()
    d3.tune_clear()


def test_long_advance_times_one_candidate_per_segment():
    d3.tune_clear()
    pool, slots = pool_with(REQS[:2], True)
    pool.advance(500)  # three segments of 100 steps time the three candidates; the rest runs at the fastest
    st = pool.tune_state()
    assert st["settled"] and st["tried"] == st["candidates"] == 3
    best = min(pool.tune_trials(), key=lambda x: x[2])
    assert (st["fluid_ctas_per_sm"], st["particle_ctas_per_sm"]) == best[:2]
    # The fluid pass: one CTA per tile (32 x 4 x 4 tiles from the lattice origin,
    # buffer layers included), the tile count rounded up by less than 1/8.
    tiles = sum(math.ceil(r.edge[0] / 32) * math.ceil(r.edge[1] / 4) * math.ceil(r.edge[2] / 4) for r in REQS[:2])
    fluid_grid = pool.get_grid()[0]
    assert tiles <= fluid_grid < tiles * 1.125 + 1
    tuned = [state(pool, s) for s in slots]
    pool.close()
    fixed, slots = pool_with(REQS[:2], False)
    fixed.advance(500)
    for s, t in zip(slots, tuned):
        bits_equal(t, state(fixed, s))
    fixed.close()
