"""BGK mode (d3q19_options.collision = 1, keyword lbm_collision 1) on the GPU.

* Against the reference's own BGK kernel collideSRT_newtonian_stream_D3Q19
  (GPU_program.cl:868-947) run with its boundary kernels in the host's step
  order (tests/golden/bgk_<case>.npz): a Couette cell with z walls over 200
  steps and a fully periodic box with a body force over 100 steps, both
  distribution layouts.  BGK here is the MRT machinery with every rate 1/tau,
  the same operator in another arithmetic order: relative L2 on u and on the
  post-boundary distributions within 1e-5 or ten times the reference's own
  spread under fused multiply-add contraction (recorded in each file),
  whichever is larger -- the rule of the golden-vector tests.  After 200
  Couette steps the reference moves u by 1.1e-5 under that change.
* Against the laws themselves: Couette flow is linear and Newtonian
  Poiseuille flow parabolic, under BGK as under MRT.
"""
import os

import numpy as np
import pytest

from cases import CASES
from gpu_helpers import REL_TOL, interior_mask, rel_l2, sim_from_golden
from test_gpu_analytic import NZ, channel, poiseuille, steady_profile, LAWS

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def load(name):
    with np.load(os.path.join(HERE, "golden", f"bgk_{name}.npz")) as z:
        return {k: z[k] for k in z.files}


@pytest.mark.parametrize("inplace", [0, 1])
@pytest.mark.parametrize("name", ["couette", "periodic_force"])
def test_bgk_matches_reference_srt_kernel(name, inplace):
    g = load(name)
    sim, ip, _ = sim_from_golden(g, CASES[name], collision=1, inplace=inplace)
    sim.run(1, int(g["iterations"]))
    sim.synchronize()
    mu, mf = interior_mask(ip, 3), interior_mask(ip, 19)
    eu = rel_l2(sim.read_u()[mu], g["final_u"][mu])
    ef = rel_l2(sim.read_f()[mf], g["final_f"][mf])
    print(name, inplace, f"u {eu:.2e} f {ef:.2e}")
    assert eu <= max(REL_TOL, 10.0 * float(g["fma_spread_u"]))
    assert ef <= max(REL_TOL, 10.0 * float(g["fma_spread_f"]))
    sim.close()


def test_bgk_differs_from_mrt():
    """The two collision operators give different flows from the same state
    (the test above would not notice a silently ignored option)."""
    g = load("couette")
    a, ip, _ = sim_from_golden(g, CASES["couette"], collision=1)
    b, _, _ = sim_from_golden(g, CASES["couette"], collision=0)
    a.run(1, 50)
    b.run(1, 50)
    mu = interior_mask(ip, 3)
    assert rel_l2(a.read_u()[mu], b.read_u()[mu]) > 1e-4
    a.close()
    b.close()


def test_bgk_couette_and_poiseuille_follow_the_laws():
    # Couette: walls +-U, linear profile (the MRT test's tolerance).
    U = 0.02
    sim = channel(1, U=U, tau=0.8, collision=1)
    u, drift = steady_profile(sim, 20000)
    sim.close()
    z = np.arange(NZ, dtype=np.float64)
    want = -U + 2.0 * U * (z - 1.0) / (NZ - 3.0)
    err = np.max(np.abs(u[1:NZ - 1] - want[1:NZ - 1])) / U
    assert err < 2e-4, err
    # Newtonian Poiseuille with body force g.
    gg = 1e-6
    law = LAWS["newtonian"]
    sim = channel(1, g=gg, tau=law["tauN"], collision=1)
    u, drift = steady_profile(sim, 80000)
    sim.close()
    u = u - 0.5 * (u[1] + u[NZ - 2])
    want = poiseuille(gg, **law)
    inner = slice(1, NZ - 1)
    err = np.max(np.abs(u[inner] - want[inner])) / np.max(want)
    assert drift < 2e-4 and err < 2e-3, (drift, err)
