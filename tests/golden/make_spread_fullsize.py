"""Rounding sensitivity of the reference itself at the sizes of the benchmarked
configurations: tests/golden/fullsize_spread.json.

For each case of tests/fullsize_cases.py the reference (oracle/_ref) runs from
its own initial state, and the oracle restatement (oracle/d3q19_oracle.c,
which reproduces the reference bit for bit without contraction) runs the same
steps from the same state compiled with fused multiply-add contraction (what
an OpenCL GPU compiler does by default).  The errors of that run against the
reference, per observable of tests/fullsize_cases.observable_errors, are how
far a benign change of FP32 arithmetic moves the reference itself after the
case's steps.  The at-size parity tests (tests/test_gpu_fullsize_parity.py)
hold the fast path to 1e-5 or to ten times this spread, whichever is larger,
the rule of the golden-vector tests (tests/golden/make_spread.py).

Usage: python tests/golden/make_spread_fullsize.py   (needs oracle/_ref and an
x86-64 CPU with FMA; a few minutes on eight cores)
"""
import ctypes as C
import json
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(REPO, "tests"))

import fullsize_cases as fc  # noqa: E402
from oracle import pyoracle as po  # noqa: E402


def main():
    if not po.ref_available():
        sys.exit("oracle/_ref is not built: run oracle/refbuild/build_ref.sh first")
    tmp = tempfile.mkdtemp()
    lib = os.path.join(tmp, "liboracle_fma.so")
    subprocess.check_call(["gcc", "-O2", "-ffp-contract=fast", "-mfma", "-mavx2", "-fopenmp", "-fPIC", "-shared",
                           "-std=gnu11", os.path.join(REPO, "oracle", "d3q19_oracle.c"), "-o", lib, "-lm"])
    po._lib = C.CDLL(lib)
    po._lib.orc_create_periodic_stream_mapping.restype = C.c_int
    po._lib.orc_tau_clamp_count.restype = C.c_longlong
    from test_oracle_pin import oracle_state  # noqa: E402

    out = {}
    for name in sorted(fc.CASES):
        case = fc.gpu_case(name)
        g = fc.reference_run(name)
        n = int(g["iterations"])
        ip, fp, st = oracle_state(po, g, case)
        st.run(1, n)
        state = {"u": st.a["u"], "f": st.latest_f(n), "tau": st.a["tau_lb"], "parKin": st.a["parKin"],
                 "parFluidForce": st.a["parFluidForce"]}
        out[name] = {"steps": n, "fma": fc.observable_errors(state, g, ip, fp, bool(case["_variable_viscosity"]))}
        print(name, {k: f"{v:.2e}" for k, v in out[name]["fma"].items()}, flush=True)
    with open(os.path.join(HERE, "fullsize_spread.json"), "w") as fh:
        json.dump(out, fh, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
