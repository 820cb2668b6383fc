"""Helpers shared by the GPU tests: build a Simulation from a golden initial
state and compare with the reference's state after N steps."""
import numpy as np

import d3q19_b200 as d3
from cases import CASES, is_variable, num_par_threads

REL_TOL = 1e-5  # relative L2 bar for floating-point results


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    if nb == 0:
        return float(np.linalg.norm(a))
    return float(np.linalg.norm(a - b) / nb)


def interior_mask(ip, comps):
    N = ip.LatticeSize
    m = np.zeros((N[2], N[1], N[0]), bool)
    m[1:-1, 1:-1, 1:-1] = True
    return np.tile(m.ravel(), comps)


def options_for(case, **over):
    o = d3.Options()
    o.variable_viscosity = int(is_variable(case))
    o.num_par_threads = num_par_threads(case)
    o.rebuild_freq = int(case.get("rebuild_neigh_list_freq", 10))
    tv = case.get("tangential_vel_bcs", (0, 0, 0))
    for d in range(3):
        o.tangential_vel_bc[d] = int(tv[d])
    for k, v in over.items():
        setattr(o, k, v)
    return o


def sim_from_golden(g, case, **over):
    ip = d3.IntParams.from_buffer_copy(bytes(g["intDat"]))
    fp = d3.FlpParams.from_buffer_copy(bytes(g["flpDat"]))
    sim = d3.Simulation(ip, fp, options_for(case, **over))
    sim.write_lattice(g["init_f"], g["init_u"], g["init_tau_lb"])
    sim.write_periodic_map(g["init_strMap"])
    if ip.NumParticles > 0:
        sim.write_particles(g["init_parKin"], g["init_parForce"], g["init_parFluidForce"], g["init_spherePoints"])
        zm = np.where(g["init_zoneMembers"] < 0, 0, g["init_zoneMembers"])
        tm = np.where(g["init_threadMembers"] < 0, 0, g["init_threadMembers"])
        sim.write_zones(g["init_zoneNeighDat"], g["init_parsZone"], zm, g["init_numParInZone"], tm,
                        g["init_numParInThread"])
    return sim, ip, fp


# The reference's compute_shear_stress quantities from a velocity field.
from fullsize_cases import shear_quantities as reference_shear  # noqa: E402,F401
