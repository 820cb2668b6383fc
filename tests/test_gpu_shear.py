"""Device-side shear diagnostics (d3q19_plane_stats, d3q19_shear_profile,
d3q19_mean_stress) through the C ABI.

* Against a float64 restatement of the same sums on the read-back u and tau
  (the device accumulates in FP64: agreement to 1e-12 relative).
* Against the reference's own compute_shear_stress quantities
  (D3Q19-OpenCL.c:670-747) evaluated on the reference's velocity field after
  N steps (the golden vectors): the wall and particle-region shear rates and
  the velocity profile within the velocity tolerance of the step.
"""
import numpy as np
import pytest

from conftest import load_golden
from cases import CASES, is_variable
from gpu_helpers import REL_TOL, reference_shear, rel_l2, sim_from_golden
from test_gpu_parity import bound

pytestmark = pytest.mark.gpu

SHEAR_CASES = ["couette", "power_law", "sphere_wrap", "contacts", "xwall_tangential", "wrap_tile_edge"]


def plane_sums(u, tau, ip, fp, variable):
    """float64 per-plane sums of the same quantities as plane_stats_kernel."""
    Nx, Ny, Nz = ip.LatticeSize
    per = [ip.BoundaryConds[d] == 0 for d in range(3)]
    U = u.astype(np.float64).reshape(3, Nz, Ny, Nx)
    T = (tau.astype(np.float64).reshape(Nz, Ny, Nx) if variable else np.full((Nz, Ny, Nx), float(fp.NewtonianTau)))

    def nb(c, d, N, periodic):
        n = c + d
        if n < 1:
            n = N - 2 if periodic else 1
        if n > N - 2:
            n = 1 if periodic else N - 2
        return n

    out = np.zeros((Nz, 5))
    xs = np.arange(1, Nx - 1)
    xm = np.array([nb(x, -1, Nx, per[0]) for x in xs])
    xp = np.array([nb(x, 1, Nx, per[0]) for x in xs])
    hx = (xp != xs).astype(float) + (xm != xs)
    for z in range(1, Nz - 1):
        zm, zp = nb(z, -1, Nz, per[2]), nb(z, 1, Nz, per[2])
        hz = (zp != z) + (zm != z)
        ys = slice(1, Ny - 1)
        dudz = (U[0, zp, ys, 1:-1] - U[0, zm, ys, 1:-1]) / hz if hz else 0.0 * U[0, z, ys, 1:-1]
        dwdx = np.where(hx > 0, (U[2, z, ys][:, xp] - U[2, z, ys][:, xm]) / np.maximum(hx, 1), 0.0)
        gxz = dudz + dwdx
        nu = (T[z, ys, 1:-1] - 0.5) / 3.0
        out[z] = [U[0, z, ys, 1:-1].sum(), U[1, z, ys, 1:-1].sum(), U[2, z, ys, 1:-1].sum(), gxz.sum(),
                  (nu * gxz).sum()]
    return out


@pytest.mark.parametrize("name", SHEAR_CASES)
def test_plane_stats_match_float64_restatement(name):
    case = CASES[name]
    g = load_golden(name)
    sim, ip, fp = sim_from_golden(g, case)
    sim.run(1, int(g["iterations"]))
    got = sim.plane_stats()
    want = plane_sums(sim.read_u(), sim.read_tau(), ip, fp, is_variable(case))
    scale = np.abs(want).max(axis=0) + 1e-30
    assert np.all(np.abs(got - want) <= 1e-12 * scale + 1e-300)
    stress, rate, visc = sim.mean_stress()
    n = (ip.LatticeSize[0] - 2) * (ip.LatticeSize[1] - 2) * (ip.LatticeSize[2] - 2)
    # Means of terms of both signs: compared to the size of the terms.
    assert abs(stress - want[:, 4].sum() / n) <= 1e-12 * np.abs(want[:, 4]).sum() / n + 1e-300
    assert abs(rate - want[:, 3].sum() / n) <= 1e-12 * np.abs(want[:, 3]).sum() / n + 1e-300
    sim.close()


@pytest.mark.parametrize("name", SHEAR_CASES)
def test_shear_profile_matches_reference_quantities(name):
    case = CASES[name]
    g = load_golden(name)
    sim, ip, fp = sim_from_golden(g, case)
    sim.run(1, int(g["iterations"]))
    mean, wall, region = sim.shear_profile()
    rmean, rwall, rregion = reference_shear(g["final_u"], ip, fp)
    # Same velocity field up to the step's parity bound for u
    # (test_gpu_parity.bound); the rates are differences of plane means, held
    # to that bound in units of the profile's largest mean speed per plane.
    tol = max(REL_TOL, bound(name, "u"))
    assert rel_l2(mean[1:-1], rmean[1:-1]) <= tol
    umax = max(np.abs(rmean[:, 0]).max(), 1e-12)
    assert abs(wall - rwall) <= tol * umax
    assert abs(region - rregion) <= tol * umax
    # And exactly the device sums' own formula on our field.
    mine = reference_shear(sim.read_u(), ip, fp)
    assert np.allclose(mean[1:-1], mine[0][1:-1], rtol=1e-12, atol=1e-18)
    assert wall == pytest.approx(mine[1], rel=1e-10, abs=1e-18)
    sim.close()
