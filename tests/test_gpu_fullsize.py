"""The full configuration sizes, held to size-independent properties
(through the C ABI).

* A fully periodic 256x128x256 box under a body force (the Casson
  configuration's lattice): streaming and collision conserve mass, and the
  Guo forcing adds exactly g per node and step to the momentum.
* The 128^3 dense suspension (200 spheres, the bench's workload) and the
  256x128x256 Casson suspension (1000 spheres, 384 markers) run without
  device errors, keep every sphere inside the lattice and every velocity
  bounded by the wall-speed scale.
"""
import os

import numpy as np
import pytest

import d3q19_b200 as d3

pytestmark = pytest.mark.gpu

C = np.array([[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1], [1, 1, 0], [1, -1, 0],
              [1, 0, 1], [1, 0, -1], [-1, 1, 0], [-1, -1, 0], [-1, 0, 1], [-1, 0, -1], [0, 1, 1], [0, 1, -1],
              [0, -1, 1], [0, -1, -1]])


def totals(f, ip):
    N = ip.LatticeSize
    nc = N[0] * N[1] * N[2]
    m = np.zeros((N[2], N[1], N[0]), bool)
    m[1:-1, 1:-1, 1:-1] = True
    m = m.ravel()
    mass, mom = 0.0, np.zeros(3)
    for q in range(19):
        s = f[q * nc:(q + 1) * nc][m].astype(np.float64).sum()
        mass += s
        mom += C[q] * s
    return mass, mom, int(m.sum())


@pytest.mark.parametrize("arith", [0, 2])
def test_periodic_box_conserves_mass_and_gains_momentum(arith):
    g = (2e-6, -1e-6, 5e-7)
    kw = dict(total_lattice_size=(256, 128, 256), boundary_conditions_xyz=(0, 0, 0), newtonian_tau=0.8,
              viscosity_model=1, constant_body_force=g, initial_vel=(0.01, 0.0, -0.005), num_particles=0)
    hs = d3.HostState(d3.parse_config(d3.keywords_text(kw)), data_dir=os.getcwd())
    sim = d3.Simulation.from_host_state(hs, arithmetic=arith)
    m0, p0, n = totals(sim.read_f(), hs.cfg.ip)
    steps = 60
    sim.run(1, steps)
    m1, p1, _ = totals(sim.read_f(), hs.cfg.ip)
    sim.close()
    # The read-back is float (the FP64 build's state rounded), which bounds
    # both checks: about 1e-8 of the mass, about 1e-4 of the momentum gain.
    assert abs(m1 - m0) <= 1e-7 * m0
    gain = p1 - p0
    want = steps * n * np.array(g)
    assert np.allclose(gain, want, rtol=2e-3, atol=0)


def suspension_clean(kw, steps, **over):
    hs = d3.HostState(d3.parse_config(d3.keywords_text(kw)), data_dir=os.getcwd())
    sim = d3.Simulation.from_host_state(hs, **over)
    sim.run(1, steps)
    sim.synchronize()  # raises on any device error (non-finite, overflow)
    ip, fp = hs.cfg.ip, hs.cfg.fp
    kin = sim.read_parkin().reshape(-1, 4)[:ip.NumParticles]
    S = np.array(ip.SystemSize, np.float64)
    assert np.all(np.isfinite(kin)) and np.all(kin[:, :3] >= 0) and np.all(kin[:, :3] < S)
    U = max(abs(v) for v in list(fp.VelUpper) + list(fp.VelLower))
    u = sim.read_u()
    assert np.all(np.isfinite(u)) and np.abs(u).max() < 10 * U
    stress, rate, visc = sim.mean_stress()
    assert np.isfinite(stress) and rate > 0 and visc > 0
    sim.close()


@pytest.mark.parametrize("storage", [0, 1])
def test_dense_suspension_128_runs_clean(storage):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    suspension_clean(bench.WORKLOADS["dense-powerlaw-128"], 400, storage=storage)


def test_casson_suspension_256x128x256_runs_clean():
    kw = dict(total_lattice_size=(256, 128, 256), boundary_conditions_xyz=(0, 0, 1), newtonian_tau=0.6,
              viscosity_model=4, viscosity_params=(1e-4, (0.6 - 0.5) / 3.0, 0.0, 0.0), use_constant_viscosity=0,
              casson_regularisation=1e-4, velocity_bc_upper=(0.04, 0.0, 0.0), velocity_bc_lower=(-0.04, 0.0, 0.0),
              num_particles=1000, particle_diameter=12.0, ibm_points_per_particle=384,
              initial_particle_distribution=4, particle_seed=1, min_particle_gap=1.0, initial_particle_buffer=0.0,
              z_wall_particle_buffer=8.0, rebuild_neigh_list_freq=10, particle_collision_params=2.0)
    suspension_clean(kw, 200)
