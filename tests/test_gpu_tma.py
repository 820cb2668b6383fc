"""The TMA-pipelined collide-stream kernel (fluid_tma_kernel, csrc/d3q19_tma.cu)
against the per-tile kernel (fluid_step_kernel): the same step, bit for bit.

A context asked for the TMA kernel (d3q19_options.fluid_kernel = 1) runs it
where its lattice allows it (periodic x and y with walls on z, the reference's
MRT, fast arithmetic, x extent a multiple of 4 nodes for FP32 and 8 for 16-bit
storage) and the per-tile kernel otherwise; fluid_kernel = 0 (the default)
runs the per-tile kernel.  Both
give the same bits: the distributions, u, tau, the sphere state, the force
partials and the zone lists, for both distribution layouts, each viscosity
law, FP32 and FP16 storage, spheres that wrap periodic edges, and a context
restored from a checkpoint at an odd in-place step (whose buffer-layer copies
the restore rebuilds from their periodic images).
"""
import numpy as np
import pytest

import d3q19_b200 as d3
from conftest import load_golden
from cases import CASES
from d3q19_b200 import serving as sv
from gpu_helpers import sim_from_golden

pytestmark = pytest.mark.gpu

TILE, TMA = 0, 1  # d3q19_options.fluid_kernel


def state(sim):
    out = {"u": sim.read_u(), "tau": sim.read_tau(), "f": sim.read_f()}
    if sim.np > 0:
        out["kin"] = sim.read_parkin()
        out["pf"] = sim.read_parforce()
        out["pff"] = sim.read_parfluidforce()
        out["zones"] = np.concatenate(sim.read_zones())
        out["cells"] = sim.read_marker_cells()
    return out


def assert_bits_equal(a, b):
    for k in a:
        x, y = np.ascontiguousarray(a[k]), np.ascontiguousarray(b[k])
        same = x.view(np.uint8) == y.view(np.uint8)
        assert x.shape == y.shape and same.all(), f"{k}: {np.count_nonzero(~same)} bytes differ"


# Golden cases whose lattice the TMA kernel takes (x extent a multiple of 4).
TMA_CASES = ["couette", "sphere_wrap", "contacts", "power_law", "power_law_half", "casson", "herschel_bulkley"]


@pytest.mark.parametrize("inplace", [0, 1])
@pytest.mark.parametrize("name", TMA_CASES)
def test_tma_kernel_matches_tile_kernel_on_golden_cases(name, inplace):
    case = CASES[name]
    g = load_golden(name)
    a, ip, _ = sim_from_golden(g, case, inplace=inplace, fluid_kernel=TMA)
    b, _, _ = sim_from_golden(g, case, inplace=inplace, fluid_kernel=TILE)
    assert a.fluid_kernel == "tma" and b.fluid_kernel == "tile"
    n = int(g["iterations"]) + 7  # odd and even step counts across the cases
    a.run(1, n)
    b.run(1, n)
    assert_bits_equal(state(a), state(b))
    a.close()
    b.close()


@pytest.mark.parametrize("over", [dict(inplace=1), dict(inplace=0), dict(inplace=1, storage=1),
                                  dict(inplace=0, storage=2)], ids=["inplace", "two-buffers", "fp16", "bf16"])
def test_tma_kernel_matches_tile_kernel_suspension(over):
    """A 64^3 power-law suspension (spheres crossing tile and periodic edges,
    zone rebuilds) over 61 steps."""
    req = sv.ShearRequest(rid=0, edge=(64, 64, 64), phi=0.2, model="power_law", wall_speed=0.04, seed=11)
    a = d3.Simulation.from_host_state(sv.host_state(req), fluid_kernel=TMA, **over)
    b = d3.Simulation.from_host_state(sv.host_state(req), fluid_kernel=TILE, **over)
    assert a.fluid_kernel == "tma" and b.fluid_kernel == "tile"
    a.run(1, 61)
    b.run(1, 61)
    assert_bits_equal(state(a), state(b))
    a.close()
    b.close()


def test_lattices_the_tma_kernel_does_not_take():
    """Fully periodic boxes, x extents that break 16-byte TMA rows, BGK,
    the reference's evaluation order and the FP64 build use the per-tile
    kernel (or the reference-order kernel)."""
    req = sv.ShearRequest(rid=0, edge=(34, 32, 32), phi=0.0, model="newtonian", wall_speed=0.02, seed=1)
    s = d3.Simulation.from_host_state(sv.host_state(req), fluid_kernel=TMA)
    assert s.fluid_kernel == "tile"  # 34 * 4 bytes is not a multiple of 16
    s.close()
    req = sv.ShearRequest(rid=0, edge=(36, 32, 32), phi=0.0, model="newtonian", wall_speed=0.02, seed=1)
    for over, want in ((dict(), "tma"), (dict(storage=1), "tile"), (dict(collision=1), "tile"),
                       (dict(arithmetic=1, periodic_smoothing=0), "reference-order"), (dict(arithmetic=2), "tile")):
        s = d3.Simulation.from_host_state(sv.host_state(req), fluid_kernel=TMA, **over)
        assert s.fluid_kernel == want, over
        s.close()
    s = d3.Simulation.from_host_state(sv.host_state(req))
    assert s.fluid_kernel == "tile"  # the default
    s.close()
    g = load_golden("periodic_force")
    s, _, _ = sim_from_golden(g, CASES["periodic_force"], fluid_kernel=TMA)
    assert s.fluid_kernel == "tile"
    s.close()


@pytest.mark.parametrize("inplace", [0, 1])
def test_restore_into_tma_context_continues_bit_for_bit(inplace):
    """A checkpoint taken after an odd number of steps (the next in-place step
    pulls from the buffer-layer copies), restored into a context that ran
    other steps, continues like the uninterrupted context -- and like the
    per-tile kernel from the same checkpoint."""
    req = sv.ShearRequest(rid=0, edge=(40, 40, 40), phi=0.15, model="casson", wall_speed=0.03, seed=5)
    a = d3.Simulation.from_host_state(sv.host_state(req), inplace=inplace, fluid_kernel=TMA)
    assert a.fluid_kernel == "tma"
    a.run(1, 23)
    ck = a.checkpoint()
    a.run(24, 20)
    want = state(a)
    a.close()
    for fk in (TMA, TILE):
        b = d3.Simulation.from_host_state(sv.host_state(req), inplace=inplace, fluid_kernel=fk)
        b.run(1, 6)
        b.restore(ck)
        b.run(24, 20)
        assert_bits_equal(want, state(b))
        b.close()
