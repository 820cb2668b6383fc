"""16-bit shifted storage of the distributions (storage = 1 FP16, 2 BF16:
f_q - w_q rounded to 16 bits once per step, FP32 arithmetic) against the
reference's FP32 state after N steps, through the C ABI.

The storage rounds each stored deviation from rest to 11 (FP16) or 8 (BF16)
significant bits every step; the tolerances below are stated per format.
They were set from the oracle with the same per-step rounding applied to its
stored distributions (FP16 / BF16: velocity rel-L2 at most 4.3e-4 / 2.3e-3 on
the Newtonian cases, 3.7e-3 / 9.9e-3 on the non-Newtonian ones; sphere
kinematics and forces in problem units at most 2e-6 / 2e-5) with margin.
"""
import numpy as np
import pytest

from conftest import load_golden
from cases import CASES, is_variable
from gpu_helpers import interior_mask, rel_l2, sim_from_golden

pytestmark = pytest.mark.gpu

# Relative L2 of u after N steps: (Newtonian, non-Newtonian) per storage.
U_TOL = {1: (1e-3, 1e-2), 2: (1e-2, 3e-2)}
# Sphere velocities, force and torque partials in units of the problem's
# scale (wall speed or peak flow speed, summed marker force at that slip).
PARTICLE_TOL = {1: 1e-4, 2: 1e-3}


def scaled_err(a, b, scale):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), scale * np.sqrt(b.size)))


@pytest.mark.parametrize("storage", [1, 2])
@pytest.mark.parametrize("name", sorted(CASES))
def test_shifted_storage_against_reference(name, storage):
    case = CASES[name]
    g = load_golden(name)
    sim, ip, fp = sim_from_golden(g, case, storage=storage)
    n = int(g["iterations"])
    sim.run(1, n)
    sim.synchronize()
    mu = interior_mask(ip, 3)
    tol = U_TOL[storage][1 if is_variable(case) else 0]
    err = rel_l2(sim.read_u()[mu], g["final_u"][mu])
    assert err <= tol, f"u rel-L2 {err:.2e} > {tol:.0e}"
    if "final_f" in g:
        mf = interior_mask(ip, 19)
        assert rel_l2(sim.read_f()[mf], g["final_f"][mf]) <= tol
    if ip.NumParticles > 0:
        np_ = ip.NumParticles
        # Velocity scale of the problem: the wall speeds, or the largest
        # velocity of the reference's flow where no wall drives it.
        U = max([abs(v) for v in list(fp.VelUpper) + list(fp.VelLower)] + [float(np.abs(g["final_u"][mu]).max()), 1e-3])
        R = fp.ParticleDiam / 2
        Fs = fp.PointArea * ip.PointsPerParticle * U / ip.WorkGroupsPerParticle
        kin = sim.read_parkin().reshape(-1, 4)
        ref = g["final_parKin"].reshape(-1, 4)
        pt = PARTICLE_TOL[storage]
        assert scaled_err(kin[np_:2 * np_, :3], ref[np_:2 * np_, :3], U) <= pt
        assert scaled_err(kin[3 * np_:, :3], ref[3 * np_:, :3], U / R) <= pt
        pff = sim.read_parfluidforce().reshape(-1, 4)
        rpff = g["final_parFluidForce"].reshape(-1, 4)
        h = pff.shape[0] // 2
        assert scaled_err(pff[:h, :3], rpff[:h, :3], Fs) <= pt
        assert scaled_err(pff[h:, :3], rpff[h:, :3], Fs * R) <= pt
        pz, _, nz = sim.read_zones()
        assert np.array_equal(pz, g["final_parsZone"]) and np.array_equal(nz, g["final_numParInZone"])
    sim.close()


def test_storage_round_trip_of_written_state():
    """write_lattice rounds to the stored form once; read_f before any step
    returns the written state to 16-bit precision of the deviation."""
    g = load_golden("couette")
    f0 = g["init_f"]
    NC = f0.size // 19
    w = np.repeat(np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12, np.float32), NC)
    for storage, eps in ((1, 2.0 ** -11), (2, 2.0 ** -8)):
        sim, _, _ = sim_from_golden(g, CASES["couette"], storage=storage)
        back = sim.read_f()
        dev = np.abs(f0 - w)
        assert np.all(np.abs(back - f0) <= eps * dev + 1e-7)
        sim.close()
