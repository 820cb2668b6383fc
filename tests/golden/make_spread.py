"""Rounding sensitivity of the reference itself: tests/golden/rounding_spread.json.

The oracle restatement reproduces the reference bit for bit when both are
evaluated without floating-point contraction (the golden vectors).  Two
benign changes of arithmetic move it away from the golden vectors, by the
amounts recorded here per case and observable as relative L2 norms:

  "fma": the same source compiled with fused multiply-add contraction (what
         an OpenCL GPU compiler does by default, FP_CONTRACT on);
  "ulp": the plain build with every stored distribution moved by a random
         -1, 0 or +1 unit in the last place after each step (two seeds, the
         larger result): a rounding difference of one ulp per value and
         step, which is what any re-implementation with different but
         correctly rounded arithmetic introduces.

They measure how well-conditioned each observable is.  Where the reference
cannot reproduce itself to 1e-5 under these changes, no re-implementation
can be held to 1e-5 either; the parity tests then use ten times the "fma"
spread or the "ulp" spread, whichever is larger (tests/test_gpu_parity.py).

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


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / nb) if nb > 0 else float(np.linalg.norm(a))


def measure(st, ip, g, case, n):
    N = list(ip.LatticeSize)
    m = np.zeros((N[2], N[1], N[0]), bool)
    m[1:-1, 1:-1, 1:-1] = True
    m1 = m.ravel()
    m3 = np.tile(m1, 3)
    d = {"u": rel(st.a["u"][m3], g["final_u"][m3]), "gpf0": rel(st.a["gpf"][: 3 * m1.size][m3], g["final_gpf0"][m3])}
    if "final_f" in g:
        m19 = np.tile(m1, 19)
        d["f"] = rel(st.latest_f(n)[m19], g["final_f"][m19])
    if is_variable(case):
        d["tau"] = rel(st.a["tau_lb"][m1], g["final_tau_lb"][m1])
        # The relaxation rate the collision consumes; tau itself is the
        # reciprocal of a noise-level strain rate at zero-shear nodes.
        d["omega"] = rel(1.0 / st.a["tau_lb"][m1], 1.0 / g["final_tau_lb"][m1])
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
    return d


def main():
    tmp = tempfile.mkdtemp()
    lib = os.path.join(tmp, "liboracle_fma.so")
    subprocess.check_call(["gcc", "-O2", "-ffp-contract=fast", "-mfma", "-mavx2", "-fopenmp", "-fPIC", "-shared",
                           "-std=gnu11", os.path.join(REPO, "oracle", "d3q19_oracle.c"), "-o", lib, "-lm"])
    plain_lib = po.lib()
    po._lib = C.CDLL(lib)
    po._lib.orc_create_periodic_stream_mapping.restype = C.c_int
    from test_oracle_pin import oracle_state  # noqa: E402
    from conftest import load_golden  # noqa: E402

    out = {}
    fma_lib = po._lib
    for name in sorted(CASES):
        case = CASES[name]
        g = load_golden(name)
        n = int(g["iterations"])
        po._lib = fma_lib
        ip, fp, st = oracle_state(po, g, case)
        st.run(1, n)
        rec = {"fma": measure(st, ip, g, case, n)}
        po._lib = plain_lib
        worst = {}
        for seed in (0, 1):
            ip, fp, st = oracle_state(po, g, case)
            rng = np.random.default_rng(seed)
            for t in range(1, n + 1):
                st.step(t)
                bits = st.latest_f(t).view(np.int32)
                bits += rng.integers(-1, 2, size=bits.shape).astype(np.int32)
            for k, v in measure(st, ip, g, case, n).items():
                worst[k] = max(worst.get(k, 0.0), v)
        rec["ulp"] = worst
        out[name] = rec
        print(name, {m: {k: f"{v:.1e}" for k, v in d.items()} for m, d in rec.items()})
    with open(os.path.join(HERE, "rounding_spread.json"), "w") as fh:
        json.dump(out, fh, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
