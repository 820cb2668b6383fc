"""Parity cases: reference input-file keyword sets for small lattices.

Each case is run through the reference itself (built from its own sources by
oracle/refbuild/build_ref.sh and executed on the host by the mock OpenCL
runtime) to produce the golden vectors in this folder (make_golden.py).  The
same keyword sets drive the oracle pin tests and the GPU parity tests.
Keyword names and meanings are the reference's (D3Q19-OpenCL.c:31-64).
"""

COMMON = dict(video_freq=1000000, shear_stress_freq=1000000, console_print_freq=1000000,
              initial_f="constant", lattice_buffer_size=(1, 1, 1), surf_point_write_atomic=8,
              particle_collision_model=1, particle_density=1.0)

CASES = {
    # Couette flow between z walls moving at +-0.02 along x; odd sizes.
    "couette": dict(COMMON, iterations=30, total_lattice_size=(12, 10, 16), boundary_conditions_xyz=(0, 0, 1),
                    newtonian_tau=0.8, viscosity_model=1, velocity_bc_upper=(0.02, 0.0, 0.0),
                    velocity_bc_lower=(-0.02, 0.0, 0.0), initial_vel=(0.01, 0.002, 0.0), num_particles=0,
                    domain_decomposition=(1, 1, 1), video_freq=15, shear_stress_freq=10, fluid_ouput_spacing=2),
    # Fully periodic box with a body force: every face/edge/vertex type.
    "periodic_force": dict(COMMON, iterations=25, total_lattice_size=(10, 12, 9), boundary_conditions_xyz=(0, 0, 0),
                           newtonian_tau=0.9, viscosity_model=1, constant_body_force=(1e-4, -2e-5, 3e-5),
                           initial_vel=(0.01, 0.005, -0.003), num_particles=0, domain_decomposition=(1, 1, 1)),
    # Walls normal to x, with the experimental tangential velocity boundary on y.
    "xwall_tangential": dict(COMMON, iterations=15, total_lattice_size=(14, 11, 9), boundary_conditions_xyz=(1, 0, 0),
                             tangential_vel_bcs=(0, 1, 0), newtonian_tau=1.1, viscosity_model=1,
                             velocity_bc_upper=(0.0, 0.03, 0.01), velocity_bc_lower=(0.0, -0.01, 0.02),
                             initial_vel=(0.0, 0.0, 0.0), num_particles=0, domain_decomposition=(1, 1, 1)),
    # One moving sphere (d=6, 128 markers) placed at x=0.5: markers wrap in x.
    "sphere_wrap": dict(COMMON, iterations=12, total_lattice_size=(20, 18, 22), boundary_conditions_xyz=(0, 0, 1),
                        newtonian_tau=0.8, viscosity_model=1, velocity_bc_upper=(0.03, 0.0, 0.0),
                        velocity_bc_lower=(-0.03, 0.0, 0.0), initial_vel=(0.0, 0.0, 0.0), num_particles=1,
                        particle_diameter=6.0, initial_particle_distribution=3, initial_particle_buffer=0.5,
                        z_wall_particle_buffer=2.0, domain_decomposition=(1, 1, 1), rebuild_neigh_list_freq=5,
                        video_freq=6, fluid_ouput_spacing=3),
    # A sphere (d=6) at the corner (0.5, 0.5, 0.5) of a fully periodic box
    # whose N-2 is a multiple of the fluid tile in every axis (32, 16, 16):
    # markers that wrap touch up to 2 x 3 x 3 = 18 tiles.  The sphere is 100
    # times denser than the fluid, so it lags the body-force driven flow and
    # its marker forces are well above rounding level.
    "wrap_tile_edge": dict(COMMON, iterations=8, total_lattice_size=(34, 18, 18), boundary_conditions_xyz=(0, 0, 0),
                           newtonian_tau=0.8, viscosity_model=1, constant_body_force=(1e-4, 0.0, 0.0),
                           initial_vel=(0.01, 0.0, 0.0), num_particles=1, particle_diameter=6.0, particle_density=100.0,
                           initial_particle_distribution=1, initial_particle_buffer=0.5, z_wall_particle_buffer=0.0,
                           domain_decomposition=(1, 1, 1), rebuild_neigh_list_freq=5),
    # Eight overlapping spheres on a grid (harmonic contact + z-wall forces),
    # two particle threads, zone rebuilds every 4 steps.
    "contacts": dict(COMMON, iterations=12, total_lattice_size=(28, 28, 30), boundary_conditions_xyz=(0, 0, 1),
                     newtonian_tau=0.8, viscosity_model=1, velocity_bc_upper=(0.02, 0.0, 0.0),
                     velocity_bc_lower=(-0.02, 0.0, 0.0), initial_vel=(0.0, 0.0, 0.0), num_particles=8,
                     particle_diameter=7.0, initial_particle_distribution=1, initial_particle_buffer=10.0,
                     z_wall_particle_buffer=11.0, domain_decomposition=(2, 1, 1), rebuild_neigh_list_freq=4,
                     particle_collision_params=2.0),
    # Jittered grid placement (unseeded rand(), D3Q19-OpenCL.c:277-279).
    "jitter": dict(COMMON, iterations=8, total_lattice_size=(26, 26, 26), boundary_conditions_xyz=(0, 0, 1),
                   newtonian_tau=0.9, viscosity_model=1, velocity_bc_upper=(0.02, 0.0, 0.0),
                   velocity_bc_lower=(-0.02, 0.0, 0.0), initial_vel=(0.0, 0.0, 0.0), num_particles=6,
                   particle_diameter=5.0, initial_particle_distribution=2, random_particle_shift=0.7,
                   initial_particle_buffer=4.0, z_wall_particle_buffer=3.0, domain_decomposition=(1, 1, 1),
                   rebuild_neigh_list_freq=3),
    # Large sphere: 1024 markers, four work-groups of 256 per sphere.
    "big_sphere": dict(COMMON, iterations=6, total_lattice_size=(22, 22, 24), boundary_conditions_xyz=(0, 0, 1),
                       newtonian_tau=0.8, viscosity_model=1, velocity_bc_upper=(0.02, 0.0, 0.0),
                       velocity_bc_lower=(-0.02, 0.0, 0.0), initial_vel=(0.0, 0.0, 0.0), num_particles=1,
                       particle_diameter=14.0, initial_particle_distribution=3, initial_particle_buffer=10.0,
                       z_wall_particle_buffer=2.0, domain_decomposition=(1, 1, 1)),
    # Power-law channel (input_file_power_law.txt geometry, shorter), built
    # without USE_CONSTANT_VISCOSITY; n=0.6 takes the pow() branch.
    "power_law": dict(COMMON, iterations=40, total_lattice_size=(8, 8, 34), boundary_conditions_xyz=(0, 0, 1),
                      constant_body_force=(1e-5, 0.0, 0.0), newtonian_tau=1.268, viscosity_model=2,
                      viscosity_params=(0.010451156235874894, 0.6, 0.0, 0.0), initial_vel=(0.0, 0.0, 0.0),
                      num_particles=0, domain_decomposition=(1, 1, 1), _variable_viscosity=True),
    "power_law_half": dict(COMMON, iterations=40, total_lattice_size=(8, 8, 34), boundary_conditions_xyz=(0, 0, 1),
                           constant_body_force=(1e-5, 0.0, 0.0), newtonian_tau=1.268, viscosity_model=2,
                           viscosity_params=(0.010451156235874894, 0.5, 0.0, 0.0), initial_vel=(0.0, 0.0, 0.0),
                           num_particles=0, domain_decomposition=(1, 1, 1), _variable_viscosity=True),
    "casson": dict(COMMON, iterations=40, total_lattice_size=(8, 8, 34), boundary_conditions_xyz=(0, 0, 1),
                   constant_body_force=(1e-5, 0.0, 0.0), newtonian_tau=1.268, viscosity_model=4,
                   viscosity_params=(0.00016, 0.0373333333333, 0.0, 0.0), initial_vel=(0.0, 0.0, 0.0),
                   num_particles=0, domain_decomposition=(1, 1, 1), _variable_viscosity=True),
    "herschel_bulkley": dict(COMMON, iterations=30, total_lattice_size=(8, 8, 30), boundary_conditions_xyz=(0, 0, 1),
                             constant_body_force=(1e-5, 0.0, 0.0), newtonian_tau=1.0, viscosity_model=3,
                             viscosity_params=(0.0001, 0.02, 0.7, 0.0), initial_vel=(0.0, 0.0, 0.0),
                             velocity_bc_upper=(0.01, 0.0, 0.0), num_particles=0, domain_decomposition=(1, 1, 1),
                             _variable_viscosity=True),
    # Power-law fluid with a moving sphere (variable-viscosity build + IBM).
    "power_law_sphere": dict(COMMON, iterations=10, total_lattice_size=(18, 18, 20), boundary_conditions_xyz=(0, 0, 1),
                             newtonian_tau=1.0, viscosity_model=2, viscosity_params=(0.03, 0.7, 0.0, 0.0),
                             velocity_bc_upper=(0.04, 0.0, 0.0), velocity_bc_lower=(-0.04, 0.0, 0.0),
                             initial_vel=(0.0, 0.0, 0.0), num_particles=1, particle_diameter=6.0,
                             initial_particle_distribution=3, initial_particle_buffer=8.0,
                             z_wall_particle_buffer=2.0, domain_decomposition=(1, 1, 1),
                             _variable_viscosity=True),
}


def input_keywords(case: dict) -> dict:
    """Keyword dict without the private (underscore) flags."""
    return {k: v for k, v in case.items() if not k.startswith("_")}


def is_variable(case: dict) -> bool:
    return bool(case.get("_variable_viscosity", False))


def num_par_threads(case: dict) -> int:
    d = case.get("domain_decomposition", (2, 2, 2))
    return int(d[0] * d[1] * d[2])
