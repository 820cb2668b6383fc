"""The FP64 forms through the C ABI.

* arithmetic = 2, the FP64 build of the fast kernels (FP64 distributions,
  collision, local tau, spread smoothing and FP64 spheres), reproduces the
  reference's state after N steps to the bounds the fast FP32 path is held
  to (tests/test_gpu_parity.py): the reference's own rounding is the
  difference.  Two cases are the exception, by construction: in a Casson or
  power-law fluid at rest the reference's local tau is the reciprocal power
  of a strain rate made of FP32 rounding noise (tau = 10.48 everywhere after
  the first step of power_law_sphere), while in FP64 the non-equilibrium part
  of the rest state is zero and the strain-rate floor 1e-8 sets tau; the
  flows then develop with different viscosities near rest.  Those two are
  held to 2e-2 in u.
* particle_precision = 1 (FP64 sphere state, force/torque sums and
  Newton-Euler integration) with the FP32 fluid, to the same bounds.
* The float read-backs are the FP64 state rounded to float.
"""
import numpy as np
import pytest

from conftest import load_golden
from cases import CASES, is_variable
from gpu_helpers import REL_TOL, interior_mask, rel_l2, sim_from_golden
from test_gpu_parity import bound, scaled_err

pytestmark = pytest.mark.gpu


# Cases whose zero-shear tau comes from FP32 rounding noise in the reference.
NOISE_TAU = {"casson", "power_law_sphere"}


def check_against_reference(name, sim, ip, fp, g, fp64=False):
    case = CASES[name]
    mu = interior_mask(ip, 3)
    if fp64 and name in NOISE_TAU:
        assert rel_l2(sim.read_u()[mu], g["final_u"][mu]) <= 2e-2
        return
    assert rel_l2(sim.read_u()[mu], g["final_u"][mu]) <= bound(name, "u")
    if is_variable(case):
        m1 = interior_mask(ip, 1)
        assert rel_l2(1.0 / sim.read_tau()[m1], 1.0 / g["final_tau_lb"][m1]) <= bound(name, "omega")
    if ip.NumParticles > 0:
        np_ = ip.NumParticles
        U = max(abs(v) for v in list(fp.VelUpper) + list(fp.VelLower) + [1e-3])
        Fscale = fp.PointArea * ip.PointsPerParticle * U
        kin = sim.read_parkin().reshape(4 * np_, 4)
        ref = g["final_parKin"].reshape(4 * np_, 4)
        assert rel_l2(kin[:np_, :3], ref[:np_, :3]) <= REL_TOL
        assert scaled_err(kin[np_:2 * np_, :3], ref[np_:2 * np_, :3], U) <= REL_TOL
        pff = sim.read_parfluidforce().reshape(-1, 4)
        rpff = g["final_parFluidForce"].reshape(-1, 4)
        half = pff.shape[0] // 2
        assert scaled_err(pff[:half, :3], rpff[:half, :3], Fscale / ip.WorkGroupsPerParticle) <= REL_TOL


@pytest.mark.parametrize("name", sorted(CASES))
def test_fp64_build_matches_reference(name):
    g = load_golden(name)
    sim, ip, fp = sim_from_golden(g, CASES[name], arithmetic=2)
    sim.run(1, int(g["iterations"]))
    sim.synchronize()
    check_against_reference(name, sim, ip, fp, g, fp64=True)
    if ip.NumParticles > 0:
        k64 = sim.read_parkin64()
        assert np.array_equal(k64.astype(np.float32), sim.read_parkin())
    sim.close()


@pytest.mark.parametrize("name", ["sphere_wrap", "contacts", "big_sphere", "jitter", "power_law_sphere",
                                  "wrap_tile_edge"])
def test_fp64_particles_match_reference(name):
    g = load_golden(name)
    sim, ip, fp = sim_from_golden(g, CASES[name], particle_precision=1)
    sim.run(1, int(g["iterations"]))
    sim.synchronize()
    check_against_reference(name, sim, ip, fp, g)
    k64 = sim.read_parkin64()
    assert np.array_equal(k64.astype(np.float32), sim.read_parkin())
    sim.close()


def test_fp64_build_is_closer_to_itself_than_fp32():
    """FP32 fast and FP64 runs of a Couette flow with a sphere agree to the
    FP32 rounding level; two FP64 runs agree bit for bit."""
    g = load_golden("sphere_wrap")
    runs = []
    for arith in (0, 2, 2):
        sim, ip, fp = sim_from_golden(g, CASES["sphere_wrap"], arithmetic=arith)
        sim.run(1, 40)
        runs.append(sim.read_u())
        sim.close()
    assert np.array_equal(runs[1], runs[2])
    assert 0 < rel_l2(runs[0], runs[1]) <= 1e-5


def test_invalid_fp64_combinations_rejected():
    import d3q19_b200 as d3
    g = load_golden("couette")
    for over in (dict(arithmetic=2, collision=1), dict(arithmetic=2, storage=1), dict(arithmetic=1, particle_precision=1)):
        with pytest.raises(d3.D3Q19Error, match="EINVAL"):
            sim_from_golden(g, CASES["couette"], **over)
