"""Generate the golden vectors in tests/golden/ from the reference itself.

Runs the reference (built from its source tree by oracle/refbuild/build_ref.sh
into oracle/_ref/ and executed on the host through the mock OpenCL runtime,
work-groups in order) for every case in cases.py, twice: with iterations=0
to capture the initial state the reference's host builds, and with the
case's iteration count to capture the state after N steps.  Buffers come
from the runtime's dump of every OpenCL buffer at release (sim_main.c:510).

Usage:  python tests/golden/make_golden.py [case ...]
Writes: tests/golden/<case>.npz
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, HERE)

from cases import CASES, input_keywords, is_variable  # noqa: E402
from oracle import pyoracle as po  # noqa: E402

MAX_F_CELLS = 12000  # store full distributions only for small lattices


def valid_members(members, counts, np_):
    out = np.full_like(members, -1)
    for z, c in enumerate(counts):
        out[z * np_: z * np_ + c] = members[z * np_: z * np_ + c]
    return out


def thread_members(members, counts, np_):
    out = np.full_like(members, -1)
    for t, c in enumerate(counts):
        out[t * np_: t * np_ + c] = members[t * np_: t * np_ + c]
    return out


def make(name):
    case = CASES[name]
    kw = input_keywords(case)
    var = is_variable(case)
    n = int(kw["iterations"])
    kw0 = dict(kw, iterations=0)
    _, b0, _ = po.run_reference(kw0, var)
    outN, bN, wd = po.run_reference(kw, var)
    a0, aN = po.ref_arrays(b0), po.ref_arrays(bN)
    ip, _ = po.params_from_bytes(bytes(a0["intDat"]), bytes(a0["flpDat"]))
    nc = ip.LatticeSize[0] * ip.LatticeSize[1] * ip.LatticeSize[2]
    np_ = ip.NumParticles
    out = {"intDat": a0["intDat"], "flpDat": a0["flpDat"], "iterations": np.int32(n),
           "variable_viscosity": np.int32(var)}
    # Initial state (both distribution buffers start equal, sim_main.c:193-194).
    out["init_f"] = a0["fB"]
    for k in ("u", "tau_lb", "strMap", "spherePoints", "zoneNeighDat", "numParInZone", "numParInThread",
              "parsZone", "parKin", "parForce", "parFluidForce"):
        out["init_" + k] = a0[k]
    out["init_zoneMembers"] = valid_members(a0["zoneMembers"], a0["numParInZone"], np_)
    out["init_threadMembers"] = thread_members(a0["threadMembers"], a0["numParInThread"], np_)
    # State after n steps: the buffer written by step n (sim_main.c:324-337).
    f_last = aN["fA"] if n % 2 == 1 else aN["fB"]
    if nc <= MAX_F_CELLS:
        out["final_f"] = f_last
    out["final_f_checksum"] = np.array([np.float64(f_last).sum(), np.float64(f_last * f_last).sum()])
    for k in ("u", "parKin", "parForce", "parFluidForce", "numParInZone", "parsZone"):
        out["final_" + k] = aN[k]
    if var:
        out["final_tau_lb"] = aN["tau_lb"]
    out["final_gpf0"] = aN["gpf"][: 3 * nc]
    out["final_zoneMembers"] = valid_members(aN["zoneMembers"], aN["numParInZone"], np_)
    out["stdout_tail"] = np.frombuffer("\n".join(outN.splitlines()[-12:]).encode(), dtype=np.uint8)
    for fn in ("velocity_field_final.txt", "xyz_ovito_output.txt", "velocity_profile_z.txt",
               "matlab_postproc/velocity_field_centerline.txt"):
        p = os.path.join(wd, fn)
        if os.path.exists(p) and os.path.getsize(p) < 400000:
            with open(p, "rb") as fh:
                out["file_" + fn.replace("/", "__")] = np.frombuffer(fh.read(), dtype=np.uint8)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    return os.path.getsize(os.path.join(HERE, name + ".npz"))


if __name__ == "__main__":
    if not po.ref_available():
        sys.exit("oracle/_ref is not built: run oracle/refbuild/build_ref.sh first")
    names = sys.argv[1:] or list(CASES)
    for nm in names:
        sz = make(nm)
        print(f"{nm}: {sz / 1024:.1f} KiB")
