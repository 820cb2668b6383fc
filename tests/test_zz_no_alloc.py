"""d3q19_read_spread_force_static, the spread force read-back that allocates
no device memory, against d3q19_read_spread_force (which grows a scratch
buffer with cudaMalloc), both through the C ABI.

Collected last so that it runs both after the other GPU tests in one process
and, alone, in a fresh one (pytest tests/test_zz_no_alloc.py)."""
import numpy as np
import pytest

from conftest import load_golden
from cases import CASES
from gpu_helpers import REL_TOL, rel_l2, sim_from_golden

import d3q19_b200 as d3

pytestmark = pytest.mark.gpu


def same_bits(a, b):
    return np.array_equal(np.ascontiguousarray(a, np.float32).view(np.uint32),
                          np.ascontiguousarray(b, np.float32).view(np.uint32))


@pytest.mark.parametrize("over", [dict(arithmetic=0), dict(arithmetic=1), dict(arithmetic=0, inplace=1)],
                         ids=["fast", "reference-order", "in-place"])
def test_static_read_back_matches_allocating_one(over):
    """Both read-backs launch the same spread kernel on the same marker lists,
    so they agree bit for bit; the in-place context ends on an odd step."""
    g = load_golden("contacts")
    sim, _, _ = sim_from_golden(g, CASES["contacts"], **over)
    sim.run(1, 5)
    first = sim.read_spread_force_static()
    second = sim.read_spread_force_static()  # two calls in a row: nothing carried over
    ref = sim.read_spread_force()
    assert np.count_nonzero(ref) > 0
    assert same_bits(first, ref)
    assert same_bits(second, ref)
    sim.run(6, 3)
    later = sim.read_spread_force_static()
    ref_later = sim.read_spread_force()
    assert same_bits(later, ref_later)
    assert rel_l2(later, ref) > REL_TOL  # the field moved on with the spheres
    sim.close()


def test_static_read_back_without_spheres_is_zero():
    g = load_golden("couette")
    sim, _, _ = sim_from_golden(g, CASES["couette"])
    sim.run(1, 2)
    for _ in range(2):
        out = sim.read_spread_force_static()
        assert out.shape == (3 * sim.nc,) and not out.any()
    sim.close()


def test_static_read_back_rejects_large_lattice():
    cfg = d3.parse_config("total_lattice_size 70 70 70\nboundary_conditions_xyz 0 0 1\nnum_particles 0\n")
    hs = d3.HostState(cfg, data_dir=".")
    sim = d3.Simulation(hs.cfg.ip, hs.cfg.fp, hs.options)
    assert sim.nc > d3.STATIC_SPREAD_MAX_CELLS
    with pytest.raises(d3.D3Q19Error, match="EINVAL.*static spread buffer"):
        sim.read_spread_force_static()
    sim.close()
