"""Pins the oracle restatement (oracle/d3q19_oracle.c) to the reference.

The golden vectors were produced by the reference itself (its own host
program and OpenCL kernels, built from source and run on the host through a
mock OpenCL runtime; tests/golden/make_golden.py).  Starting from the
reference's initial state, the oracle must reproduce the reference's state
after N steps bit for bit: the restatement follows the reference's
floating-point evaluation order term for term.
"""
import numpy as np
import pytest

from conftest import load_golden
from cases import CASES, is_variable, num_par_threads

ARRAYS = ["u", "tau_lb", "strMap", "spherePoints", "zoneNeighDat", "numParInZone", "numParInThread", "parsZone",
          "parKin", "parForce", "parFluidForce", "zoneMembers", "threadMembers"]


def oracle_state(po, g, case):
    ip, fp = po.params_from_bytes(bytes(g["intDat"]), bytes(g["flpDat"]))
    nc = ip.LatticeSize[0] * ip.LatticeSize[1] * ip.LatticeSize[2]
    a = {k: g["init_" + k] for k in ARRAYS}
    a["fA"] = g["init_f"].copy()
    a["fB"] = g["init_f"].copy()
    a["gpf"] = np.zeros(3 * ip.MaxSurfPointsPerNode * nc, np.float32)
    a["countPoint"] = np.zeros(nc, np.int32)
    # Entries past each zone's count are the reference's uninitialised malloc
    # tail; they are never read.
    a["zoneMembers"] = np.where(a["zoneMembers"] < 0, 0, a["zoneMembers"]).astype(np.int32)
    a["threadMembers"] = np.where(a["threadMembers"] < 0, 0, a["threadMembers"]).astype(np.int32)
    st = po.OracleState(ip, fp, a, num_par_threads(case), int(case.get("rebuild_neigh_list_freq", 10)),
                        is_variable(case), tuple(case.get("tangential_vel_bcs", (0, 0, 0))))
    return ip, fp, st


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_reference_bitwise(oracle_lib, name):
    po = oracle_lib
    case = CASES[name]
    g = load_golden(name)
    ip, fp, st = oracle_state(po, g, case)
    n = int(g["iterations"])
    st.run(1, n)
    f = st.latest_f(n)
    if "final_f" in g:
        assert np.array_equal(f.view(np.uint32), g["final_f"].view(np.uint32))
    ck = g["final_f_checksum"]
    assert np.float64(f).sum() == ck[0] and np.float64(f * f).sum() == ck[1]
    assert np.array_equal(st.a["u"].view(np.uint32), g["final_u"].view(np.uint32))
    nc = ip.LatticeSize[0] * ip.LatticeSize[1] * ip.LatticeSize[2]
    assert np.array_equal(st.a["gpf"][: 3 * nc].view(np.uint32), g["final_gpf0"].view(np.uint32))
    if is_variable(case):
        assert np.array_equal(st.a["tau_lb"].view(np.uint32), g["final_tau_lb"].view(np.uint32))
    for k in ("parKin", "parForce", "parFluidForce"):
        assert np.array_equal(st.a[k].view(np.uint32), g["final_" + k].view(np.uint32)), k
    assert np.array_equal(st.a["numParInZone"], g["final_numParInZone"])
    assert np.array_equal(st.a["parsZone"], g["final_parsZone"])
    zm = g["final_zoneMembers"]
    valid = zm >= 0
    assert np.array_equal(st.a["zoneMembers"][valid], zm[valid])


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_periodic_map_and_zone_table(oracle_lib, name):
    import ctypes as C
    po = oracle_lib
    g = load_golden(name)
    ip, fp = po.params_from_bytes(bytes(g["intDat"]), bytes(g["flpDat"]))
    nc = ip.LatticeSize[0] * ip.LatticeSize[1] * ip.LatticeSize[2]
    sm = np.zeros(2 * nc, np.int32)
    n = po.lib().orc_create_periodic_stream_mapping(C.byref(ip), sm.ctypes.data_as(C.c_void_p))
    assert np.array_equal(sm[: 2 * n], g["init_strMap"])
    nz = ip.NumZones[0] * ip.NumZones[1] * ip.NumZones[2]
    znd = np.zeros(28 * nz, np.int32)
    po.lib().orc_zone_neighbours(C.byref(ip), znd.ctypes.data_as(C.c_void_p))
    ref = g["init_zoneNeighDat"]
    for z in range(nz):  # entries past the count are calloc'ed zeros in the reference
        cnt = ref[28 * z]
        assert np.array_equal(znd[28 * z: 28 * z + 1 + cnt], ref[28 * z: 28 * z + 1 + cnt])
