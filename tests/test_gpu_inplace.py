"""In-place streaming (d3q19_options.inplace = 1, the AA pattern) on the GPU.

One distribution buffer instead of two: even steps read a node's own cells
and write them back with the directions reversed; odd steps pull the
reversed cells of the upwind neighbours and push to the downwind ones.  The
arithmetic is the two-buffer step's, so every result must be bit-identical
to it: on every boundary layout (periodic, z walls, x walls with tangential
velocity), with spheres, contacts and each viscosity law, in FP32, FP16
storage and the FP64 build, stepped one by one or replayed as graphs, and
across checkpoints taken at either phase.
"""
import numpy as np
import pytest

import d3q19_b200 as d3
from cases import CASES
from conftest import load_golden
from gpu_helpers import sim_from_golden

pytestmark = pytest.mark.gpu

NAMES = ["couette", "periodic_force", "xwall_tangential", "sphere_wrap", "wrap_tile_edge", "contacts",
         "power_law", "casson", "herschel_bulkley", "power_law_sphere"]


def state(sim):
    out = {"u": sim.read_u(), "tau": sim.read_tau(), "f": sim.read_f()}
    if sim.np > 0:
        out["kin"] = sim.read_parkin()
        out["pff"] = sim.read_parfluidforce()
        out["gpf"] = sim.read_spread_force()
    return out


def bits_equal(a, b):
    for k in a:
        x, y = np.ascontiguousarray(a[k]), np.ascontiguousarray(b[k])
        assert x.shape == y.shape and np.array_equal(x.view(np.uint8), y.view(np.uint8)), k


def run_case(name, inplace, steps, by_step=False, **over):
    g = load_golden(name)
    sim, _, _ = sim_from_golden(g, CASES[name], inplace=inplace, **over)
    if by_step:
        for t in range(1, steps + 1):
            sim.step(t)
    else:
        sim.run(1, steps)
    out = state(sim)
    sim.close()
    return out


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("steps", [7, 12])
def test_inplace_matches_two_buffers(name, steps):
    bits_equal(run_case(name, 0, steps), run_case(name, 1, steps))


@pytest.mark.parametrize("over", [dict(storage=1), dict(arithmetic=2)], ids=["fp16", "fp64-build"])
@pytest.mark.parametrize("name", ["sphere_wrap", "power_law"])
def test_inplace_other_precisions(name, over):
    bits_equal(run_case(name, 0, 9, **over), run_case(name, 1, 9, **over))


def test_inplace_step_by_step_matches_graphs():
    bits_equal(run_case("contacts", 1, 11, by_step=True), run_case("contacts", 1, 11))


@pytest.mark.parametrize("at", [6, 7])
def test_inplace_checkpoint_at_either_phase(at):
    g = load_golden("sphere_wrap")
    a, _, _ = sim_from_golden(g, CASES["sphere_wrap"], inplace=1)
    a.run(1, at)
    ck = a.checkpoint()
    a.run(at + 1, 10)
    want = state(a)
    a.close()
    b, _, _ = sim_from_golden(g, CASES["sphere_wrap"], inplace=1)
    b.run(1, 3)  # another phase, overwritten by the restore
    b.restore(ck)
    b.run(at + 1, 10)
    bits_equal(want, state(b))
    b.close()
    # A two-buffer context does not take an in-place checkpoint.
    c, _, _ = sim_from_golden(g, CASES["sphere_wrap"], inplace=0)
    with pytest.raises(d3.D3Q19Error, match="EINVAL"):
        c.restore(ck)
    c.close()


def test_inplace_memory_and_refusals():
    g = load_golden("contacts")
    ip = d3.IntParams.from_buffer_copy(bytes(g["intDat"]))
    o0, o1 = d3.Options(), d3.Options()
    o1.inplace = 1
    nc = ip.LatticeSize[0] * ip.LatticeSize[1] * ip.LatticeSize[2]
    saved = d3.context_bytes(ip, o0) - d3.context_bytes(ip, o1)
    assert 19 * 4 * nc <= saved <= 19 * 4 * nc + 4096
    with pytest.raises(d3.D3Q19Error, match="EINVAL"):
        sim_from_golden(g, CASES["contacts"], inplace=1, arithmetic=1)
    from d3q19_b200 import serving as sv

    # The members of a pool share one layout.
    pool = d3.Pool(storage=0, max_slots=2)
    req = sv.ShearRequest(rid=0, edge=(32, 32, 32), phi=0.1, model="newtonian", wall_speed=0.02, seed=3)
    s = pool.admit(sv.host_state(req))
    with pytest.raises(d3.D3Q19Error, match="EINVAL"):
        pool.admit(sv.host_state(req), inplace=1)
    pool.release(s)
    assert pool.admit(sv.host_state(req), inplace=1) is not None  # an empty pool takes either
    pool.close()
