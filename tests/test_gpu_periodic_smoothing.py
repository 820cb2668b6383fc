"""Periodic smoothing of the spread force (d3q19_options.periodic_smoothing,
keyword periodic_force_smoothing; the reference's smoothing is the default).

The reference smooths the spread force with its 27-point stencil reading the
buffer layer as zero, without wrapping across periodic axes
(GPU_program.cl:356-377).  A sphere on a periodic seam then loses the part of
its reaction on the fluid that the smoothing would carry across the seam.

* Momentum balance (FP64 build): a sphere held fixed across the periodic x
  seam of a fully periodic box, the fluid driven by a body force g.  At steady
  state the fluid's momentum is constant, so the force the markers apply to
  the fluid balances g on every node.  With the smoothing wrapped, the sum of
  the marker forces equals g N to 1e-6; with the reference's smoothing the
  markers must push harder to make up for the lost part, and the sum exceeds
  g N by far more.
* Regression: request 70 of the served sweep's arrivals (seed 2024; Newtonian,
  60^3, phi 0.264) went non-finite in FP16 storage after about 19,500 steps
  with the reference's smoothing: the fluid on the seams reached 0.2-0.44
  (0.22 in FP32) against a wall speed of 0.02.  With the smoothing wrapped it
  stays finite over 20,000 steps and no node moves faster than the walls by
  more than half their speed.
"""
import numpy as np
import pytest

import d3q19_b200 as d3
from d3q19_b200 import serving as sv

pytestmark = pytest.mark.gpu


def seam_sphere_balance(periodic_smoothing, L=34, g=1e-5, d=8.0, steps=40000):
    """(sum of the marker forces along x, its change over the last 5000 steps,
    g times the interior nodes) for a sphere fixed at x = 0.5 (across the seam)
    in a fully periodic L^3 box, FP64 build."""
    S = L - 2
    kw = dict(iterations=10 ** 6, total_lattice_size=(L, L, L), boundary_conditions_xyz=(0, 0, 0),
              newtonian_tau=1.0, viscosity_model=1, use_constant_viscosity=1, constant_body_force=(g, 0.0, 0.0),
              initial_f="constant", initial_vel=(0.0, 0.0, 0.0), domain_decomposition=(1, 1, 1), num_particles=1,
              particle_diameter=d, initial_particle_distribution=3, initial_particle_buffer=0.5,
              fixed_particles=1, rebuild_neigh_list_freq=10, video_freq=10 ** 9, shear_stress_freq=10 ** 9,
              console_print_freq=10 ** 9, periodic_force_smoothing=periodic_smoothing)
    sim = d3.Simulation.from_host_state(d3.HostState(d3.parse_config(d3.keywords_text(kw))), arithmetic=2)

    def force():
        pff = sim.read_parfluidforce().reshape(2, sim.np, sim.nfa, 4).astype(np.float64)
        return float(pff[0, 0, :, 0].sum())

    # The direct-forcing feedback alternates slightly from step to step: the
    # balance is taken on the mean of two steps.
    sim.run(1, steps - 5000)
    f0 = force()
    sim.run(steps - 4999, 5000)
    f1 = force()
    sim.run(steps + 1, 1)
    f1 = 0.5 * (f1 + force())
    sim.close()
    return f1, abs(f1 - f0) / abs(f1), g * S ** 3


def test_wrapped_smoothing_balances_momentum_across_the_seam():
    f_wrap, drift_wrap, gN = seam_sphere_balance(1)
    f_ref, drift_ref, _ = seam_sphere_balance(0)
    e_wrap = abs(f_wrap - gN) / gN
    e_ref = abs(f_ref - gN) / gN
    print(f"seam sphere: wrapped {e_wrap:.2e} (drift {drift_wrap:.1e}), reference smoothing {e_ref:.2e}")
    assert drift_wrap < 1e-5 and e_wrap < 1e-6
    assert e_ref > 100 * max(e_wrap, 1e-8)


def test_dense_served_suspension_stays_finite_in_fp16():
    req = [r for r in sv.make_requests(128, 50.0, 2024, edges=(32, 64)) if r.rid == 70][0]
    assert req.model == "newtonian" and req.edge == (60, 60, 60)
    kw = sv.solve_keywords(req)
    assert kw["periodic_force_smoothing"] == 1
    s = d3.Simulation.from_host_state(sv.host_state(req), storage=1, inplace=1)
    vmax = 0.0
    for t in range(1, 20001, 2000):
        s.run(t, 2000)  # raises D3Q19Error (ENUMERIC) on a non-finite state
        vmax = max(vmax, float(np.abs(s.read_u()).max()))
    s.close()
    assert vmax <= 1.5 * req.wall_speed, vmax
