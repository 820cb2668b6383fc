"""The precision claim against the FP64 build (d3q19_options.arithmetic = 2):
16-bit shifted storage of the distributions with FP32 arithmetic keeps the
suspension's effective viscosity within 1e-3 of the FP64 build.

Workload: the Casson suspension of the precision study (regularised yield
stress 1e-4, plastic tau 0.6, walls +-0.04, spheres of radius 6 with 384
markers, seeded random placement) on a 96 x 64 x 96 lattice with 100 spheres
(volume fraction 0.2 of the box), 2000 steps; each storage form runs the same
steps from the same initial state as the FP64 build.  Checked: effective
viscosity and mean shear stress (FP64 device sums over the interior) within
1e-3 for FP32 and FP16 storage, and u within 1e-3 relative L2.  BF16 storage
(8-bit significand) is recorded and held only to 1e-2 (u to 5e-2): it does not meet the
1e-3 bound on the effective viscosity (measured 2.4e-3 on the full-size
study), and the library documents it as such.
"""
import numpy as np
import pytest

import d3q19_b200 as d3

pytestmark = pytest.mark.gpu

KW = dict(iterations=2000, total_lattice_size=(96, 64, 96), boundary_conditions_xyz=(0, 0, 1),
          newtonian_tau=0.6, viscosity_model=4, viscosity_params=(1e-4, (0.6 - 0.5) / 3.0, 0.0, 0.0),
          use_constant_viscosity=0, casson_regularisation=1e-4, velocity_bc_upper=(0.04, 0.0, 0.0),
          velocity_bc_lower=(-0.04, 0.0, 0.0), initial_f="constant", initial_vel=(0.0, 0.0, 0.0),
          num_particles=100, particle_diameter=12.0, ibm_points_per_particle=384,
          initial_particle_distribution=4, particle_seed=3, min_particle_gap=1.0, initial_particle_buffer=0.0,
          z_wall_particle_buffer=8.0, domain_decomposition=(1, 1, 1), rebuild_neigh_list_freq=10,
          particle_collision_params=2.0, video_freq=10 ** 9, shear_stress_freq=10 ** 9, console_print_freq=10 ** 9)

# storage form -> bound on the effective viscosity and mean stress errors
BOUND = {"fp32": 1e-3, "fp16": 1e-3, "bf16": 1e-2}
U_BOUND = {"fp32": 1e-3, "fp16": 1e-3, "bf16": 5e-2}
OVER = {"fp64": dict(arithmetic=2), "fp32": {}, "fp16": dict(storage=1), "bf16": dict(storage=2)}

_RESULTS = {}


def run(label):
    if label not in _RESULTS:
        hs = d3.HostState(d3.parse_config(d3.keywords_text(KW)))
        sim = d3.Simulation.from_host_state(hs, **OVER[label])
        sim.run(1, KW["iterations"])
        _RESULTS[label] = dict(u=sim.read_u().astype(np.float64), stress=sim.mean_stress())
        sim.close()
    return _RESULTS[label]


@pytest.mark.parametrize("label", ["fp32", "fp16", "bf16"])
def test_storage_form_against_fp64_build(label):
    ref, got = run("fp64"), run(label)
    e_visc = abs(got["stress"][2] - ref["stress"][2]) / abs(ref["stress"][2])
    e_stress = abs(got["stress"][0] - ref["stress"][0]) / abs(ref["stress"][0])
    e_u = float(np.linalg.norm(got["u"] - ref["u"]) / np.linalg.norm(ref["u"]))
    print(f"{label}: effective viscosity {e_visc:.2e}, mean stress {e_stress:.2e}, u {e_u:.2e}")
    assert e_visc <= BOUND[label] and e_stress <= BOUND[label]
    assert e_u <= U_BOUND[label]
