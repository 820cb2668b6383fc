"""Rounding sensitivity of the reference itself: tests/golden/rounding_spread.json.

The oracle restatement reproduces the reference bit for bit when both are
evaluated without floating-point contraction (the golden vectors).  Compiled
with fused multiply-add contraction -- what an OpenCL GPU compiler does by
default (FP_CONTRACT on) -- the same source gives results that differ from
the golden vectors by the amounts recorded here, per case and observable, as
relative L2 norms.  They measure how well-conditioned each observable is:
where the reference cannot reproduce itself to 1e-5 under that benign change,
no re-implementation can be held to 1e-5 either, and the parity tests use
ten times this spread instead (tests/test_gpu_parity.py).

Usage: python tests/golden/make_spread.py   (needs an x86-64 CPU with FMA)
"""
import ctypes as C
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(REPO, "tests"))

from cases import CASES, is_variable  # noqa: E402
from oracle import pyoracle as po  # noqa: E402


def observables(st, ip, g_final_like):
    return st


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / nb) if nb > 0 else float(np.linalg.norm(a))


def main():
    tmp = tempfile.mkdtemp()
    lib = os.path.join(tmp, "liboracle_fma.so")
    subprocess.check_call(["gcc", "-O2", "-ffp-contract=fast", "-mfma", "-mavx2", "-fopenmp", "-fPIC", "-shared",
                           "-std=gnu11", os.path.join(REPO, "oracle", "d3q19_oracle.c"), "-o", lib, "-lm"])
    po._lib = C.CDLL(lib)
    po._lib.orc_create_periodic_stream_mapping.restype = C.c_int
    from test_oracle_pin import oracle_state  # noqa: E402
    from conftest import load_golden  # noqa: E402

    out = {}
    for name in sorted(CASES):
        case = CASES[name]
        g = load_golden(name)
        ip, fp, st = oracle_state(po, g, case)
        n = int(g["iterations"])
        st.run(1, n)
        N = list(ip.LatticeSize)
        m = np.zeros((N[2], N[1], N[0]), bool)
        m[1:-1, 1:-1, 1:-1] = True
        m1 = m.ravel()
        m3 = np.tile(m1, 3)
        d = {"u": rel(st.a["u"][m3], g["final_u"][m3]), "gpf0": rel(st.a["gpf"][: 3 * m1.size][m3],
                                                                        g["final_gpf0"][m3])}
        if "final_f" in g:
            m19 = np.tile(m1, 19)
            d["f"] = rel(st.latest_f(n)[m19], g["final_f"][m19])
        if is_variable(case):
            d["tau"] = rel(st.a["tau_lb"][m1], g["final_tau_lb"][m1])
        npp = ip.NumParticles
        if npp:
            k, r = st.a["parKin"].reshape(-1, 4), g["final_parKin"].reshape(-1, 4)
            d["position"] = rel(k[:npp, :3], r[:npp, :3])
            d["velocity"] = rel(k[npp:2 * npp, :3], r[npp:2 * npp, :3])
            d["angular_velocity"] = rel(k[3 * npp:, :3], r[3 * npp:, :3])
            pf, rp = st.a["parFluidForce"].reshape(-1, 4), g["final_parFluidForce"].reshape(-1, 4)
            h = len(pf) // 2
            d["force_partials"] = rel(pf[:h, :3], rp[:h, :3])
            d["torque_partials"] = rel(pf[h:, :3], rp[h:, :3])
            f1, r1 = st.a["parForce"].reshape(-1, 4), g["final_parForce"].reshape(-1, 4)
            d["particle_force"] = rel(f1[:npp, :3], r1[:npp, :3])
        out[name] = d
        print(name, {k: f"{v:.1e}" for k, v in d.items()})
    with open(os.path.join(HERE, "rounding_spread.json"), "w") as fh:
        json.dump(out, fh, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
