"""Parity cases at the sizes of the benchmarked configurations, as the
reference's input files express them, the reference's own runs of them, and
the observables compared.

The reference (its unmodified host program and OpenCL kernels, built for the
host cores into oracle/_ref by oracle/refbuild/build_ref.sh and run through the
mock OpenCL runtime) runs each case from the initial state its host builds.
The IBM kernel runs its work-groups in order (MOCKCL_SERIAL_FIBERS): its
slot updates race between concurrent work-groups, the other kernels run in
parallel over the host cores.

Cases (keyword names and meanings are the reference's, D3Q19-OpenCL.c:31-64):
* couette_sphere_64: the 64^3 Couette cell (walls +-0.02, Newtonian tau 0.8)
  with one sphere of diameter 16 at the box centre, 2000 steps; the reference
  derives 1024 markers for d = 16 and integrates the sphere.
* suspension_128: the 128^3 power-law suspension (n = 0.6, walls +-0.05) with
  200 spheres of diameter 16 on the reference's jittered grid, 1024 markers
  each, 30 steps (the reference's build without USE_CONSTANT_VISCOSITY).
"""
import numpy as np

COMMON = dict(video_freq=1000000, shear_stress_freq=1000000, console_print_freq=1000000, initial_f="constant",
              lattice_buffer_size=(1, 1, 1), surf_point_write_atomic=8, particle_collision_model=1,
              particle_density=1.0, initial_vel=(0.0, 0.0, 0.0))

CASES = {
    "couette_sphere_64": dict(
        COMMON, iterations=2000, total_lattice_size=(64, 64, 64), boundary_conditions_xyz=(0, 0, 1),
        newtonian_tau=0.8, viscosity_model=1, velocity_bc_upper=(0.02, 0.0, 0.0), velocity_bc_lower=(-0.02, 0.0, 0.0),
        num_particles=1, particle_diameter=16.0, initial_particle_distribution=3, initial_particle_buffer=31.0,
        z_wall_particle_buffer=2.0, domain_decomposition=(1, 1, 1), rebuild_neigh_list_freq=10),
    "suspension_128": dict(
        COMMON, iterations=30, total_lattice_size=(128, 128, 128), boundary_conditions_xyz=(0, 0, 1),
        newtonian_tau=1.0, viscosity_model=2, viscosity_params=(0.0105, 0.6, 0.0, 0.0),
        velocity_bc_upper=(0.05, 0.0, 0.0), velocity_bc_lower=(-0.05, 0.0, 0.0), num_particles=200,
        particle_diameter=16.0, initial_particle_distribution=2, random_particle_shift=0.5,
        initial_particle_buffer=8.0, z_wall_particle_buffer=2.0, domain_decomposition=(1, 1, 1),
        rebuild_neigh_list_freq=10, particle_collision_params=2.0, _variable_viscosity=True),
}


def keywords(name):
    """(input-file keywords, variable-viscosity build) of a case."""
    kw = {k: v for k, v in CASES[name].items() if not k.startswith("_")}
    return kw, bool(CASES[name].get("_variable_viscosity", False))


def gpu_case(name):
    """The case in the form the GPU helpers read (tests/gpu_helpers.py)."""
    kw, var = keywords(name)
    return dict(kw, _variable_viscosity=var)


_RUNS = {}


def reference_run(name):
    """Initial state and the state after the case's steps from the reference
    itself, in the layout of the golden vectors (cached per process)."""
    if name in _RUNS:
        return _RUNS[name]
    from oracle import pyoracle as po

    kw, var = keywords(name)
    env = {"MOCKCL_SERIAL_FIBERS": "1"}
    n = int(kw["iterations"])
    _, b0, _ = po.run_reference(dict(kw, iterations=0), var, serial=False, extra_env=env)
    _, bN, _ = po.run_reference(kw, var, serial=False, extra_env=env)
    a0, aN = po.ref_arrays(b0), po.ref_arrays(bN)
    ip, _ = po.params_from_bytes(bytes(a0["intDat"]), bytes(a0["flpDat"]))
    np_ = ip.NumParticles

    def valid(members, counts):
        out = np.full_like(members, -1)
        for z, c in enumerate(counts):
            out[z * np_: z * np_ + c] = members[z * np_: z * np_ + c]
        return out

    g = {"intDat": a0["intDat"], "flpDat": a0["flpDat"], "iterations": n, "init_f": a0["fB"]}
    for k in ("u", "tau_lb", "strMap", "spherePoints", "zoneNeighDat", "numParInZone", "numParInThread", "parsZone",
              "parKin", "parForce", "parFluidForce"):
        g["init_" + k] = a0[k]
    g["init_zoneMembers"] = valid(a0["zoneMembers"], a0["numParInZone"])
    g["init_threadMembers"] = valid(a0["threadMembers"], a0["numParInThread"])
    g["final_f"] = aN["fA"] if n % 2 == 1 else aN["fB"]
    for k in ("u", "parKin", "parForce", "parFluidForce", "numParInZone", "parsZone", "tau_lb"):
        g["final_" + k] = aN[k]
    g["final_zoneMembers"] = valid(aN["zoneMembers"], aN["numParInZone"])
    g["final_gpf0"] = aN["gpf"][: 3 * ip.LatticeSize[0] * ip.LatticeSize[1] * ip.LatticeSize[2]]
    _RUNS[name] = g
    return g


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / nb) if nb > 0 else float(np.linalg.norm(a))


def scaled_err(a, b, scale):
    """L2 error relative to max(|b|, a scale per entry)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), scale * np.sqrt(b.size)))


def shear_quantities(u, ip, fp):
    """The reference's compute_shear_stress quantities (D3Q19-OpenCL.c:
    670-747) of a velocity field: plane means, wall and particle-region
    shear rates."""
    Nx, Ny, Nz = ip.LatticeSize
    U = u.astype(np.float64).reshape(3, Nz, Ny, Nx)
    nxy = (Nx - 2) * (Ny - 2)
    mean = np.array([[U[d, z, 1:-1, 1:-1].sum() / nxy for d in range(3)] for z in range(Nz)])
    dz, zA, zB = 4, 6, Nz - 3
    s = 0.0
    if 1 <= zA <= Nz - 2:
        s += (U[0, zA, 1:-1, 1:-1] - U[0, zA - dz, 1:-1, 1:-1]).sum() / dz
    if zB != zA and 1 <= zB <= Nz - 2 and zB - dz >= 0:
        s += (U[0, zB, 1:-1, 1:-1] - U[0, zB - dz, 1:-1, 1:-1]).sum() / dz
    wall = s / (2.0 * nxy)
    ib = int(fp.ParticleZBuffer + 1e-8) + int(fp.ParticleDiam / 2)
    zbL, zbU = 1 + ib, Nz - 2 - ib
    ok = 0 <= zbL < Nz and 0 <= zbU < Nz and zbU != zbL
    region = (mean[zbU, 0] - mean[zbL, 0]) / (zbU - zbL) if ok else 0.0
    return mean, wall, region


def observable_errors(state, g, ip, fp, variable):
    """Errors of a final state against the reference's, by observable.

    state: u, f (post-boundary, the reference's layout), tau, parKin,
    parFluidForce, parForce as flat float arrays.  Sphere velocities and force
    partials are compared in the problem's own units (wall speed U, summed
    marker force at slip U), as test_gpu_parity does: after a few steps they
    are residuals of nearly cancelling marker forces.  The shear rates are
    held in units of the profile's largest plane-mean speed."""
    N = list(ip.LatticeSize)
    m = np.zeros((N[2], N[1], N[0]), bool)
    m[1:-1, 1:-1, 1:-1] = True
    m1 = m.ravel()
    m3, m19 = np.tile(m1, 3), np.tile(m1, 19)
    e = {"u": rel_l2(state["u"][m3], g["final_u"][m3]), "f": rel_l2(state["f"][m19], g["final_f"][m19])}
    if variable:
        e["omega"] = rel_l2(1.0 / state["tau"][m1], 1.0 / g["final_tau_lb"][m1])
    np_ = ip.NumParticles
    U = max(abs(v) for v in list(fp.VelUpper) + list(fp.VelLower))
    R = fp.ParticleDiam / 2
    Fscale = fp.PointArea * ip.PointsPerParticle * U
    kin = state["parKin"].reshape(4 * np_, 4)
    ref = g["final_parKin"].reshape(4 * np_, 4)
    e["position"] = rel_l2(kin[:np_, :3], ref[:np_, :3])
    e["velocity"] = scaled_err(kin[np_:2 * np_, :3], ref[np_:2 * np_, :3], U)
    e["angular"] = scaled_err(kin[3 * np_:, :3], ref[3 * np_:, :3], U / R)
    pff = state["parFluidForce"].reshape(-1, 4)
    rpff = g["final_parFluidForce"].reshape(-1, 4)
    half = pff.shape[0] // 2
    e["force"] = scaled_err(pff[:half, :3], rpff[:half, :3], Fscale / ip.WorkGroupsPerParticle)
    e["torque"] = scaled_err(pff[half:, :3], rpff[half:, :3], Fscale * R / ip.WorkGroupsPerParticle)
    mean, wall, region = shear_quantities(state["u"], ip, fp)
    rmean, rwall, rregion = shear_quantities(g["final_u"], ip, fp)
    umax = max(np.abs(rmean[:, 0]).max(), 1e-12)
    e["profile"] = rel_l2(mean[1:-1], rmean[1:-1])
    e["wall_rate"] = abs(wall - rwall) / umax
    e["region_rate"] = abs(region - rregion) / umax
    return e
