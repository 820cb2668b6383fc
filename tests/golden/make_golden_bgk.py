"""BGK golden vectors from the reference itself: tests/golden/bgk_<case>.npz.

The reference's BGK kernel collideSRT_newtonian_stream_D3Q19
(GPU_program.cl:868-947), which its host program does not call, runs with the
reference's periodic and velocity boundary kernels in the host's per-step
order (oracle/refbuild/srt_driver.c, built by oracle/refbuild/build_ref.sh into
oracle/_ref) from the initial state of a golden case (the reference host's
own initial lattice).  The kernel takes its body force from a force field;
ConstBodyForce is given at every node (a fluid without spheres).  Each file
also records how far the same kernels compiled with fused multiply-add
contraction move u and f (the reference's own rounding spread).

Usage:  python tests/golden/make_golden_bgk.py
Writes: tests/golden/bgk_<case>.npz
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, HERE)

from oracle import pyoracle as po  # noqa: E402

# golden case -> steps of the BGK run
BGK_CASES = {"couette": 200, "periodic_force": 100}


def srt_inputs(g):
    ip = po.IntParams.from_buffer_copy(bytes(g["intDat"]))
    fp = po.FlpParams.from_buffer_copy(bytes(g["flpDat"]))
    nc = ip.LatticeSize[0] * ip.LatticeSize[1] * ip.LatticeSize[2]
    force = np.repeat(np.array(list(fp.ConstBodyForce), np.float32), nc)
    return bytes(g["intDat"]), bytes(g["flpDat"]), g["init_f"], force, g["init_strMap"]


def make(name, steps):
    with np.load(os.path.join(HERE, name + ".npz")) as z:
        g = {k: z[k] for k in z.files}
    ib, fb, f0, force, sm = srt_inputs(g)
    f, u = po.run_srt(ib, fb, f0, force, sm, steps)
    # The reference's own rounding spread: the same kernels with fused
    # multiply-add contraction, relative L2 over the interior.
    ff, uf = po.run_srt(ib, fb, f0, force, sm, steps, fma=True)
    ip = po.IntParams.from_buffer_copy(ib)
    N = list(ip.LatticeSize)
    m = np.zeros((N[2], N[1], N[0]), bool)
    m[1:-1, 1:-1, 1:-1] = True
    m3, m19 = np.tile(m.ravel(), 3), np.tile(m.ravel(), 19)

    def rel(a, b):
        return np.linalg.norm(np.float64(a) - np.float64(b)) / np.linalg.norm(np.float64(b))

    out = {"case": np.frombuffer(name.encode(), np.uint8), "intDat": g["intDat"], "flpDat": g["flpDat"],
           "init_f": f0, "init_u": g["init_u"], "init_tau_lb": g["init_tau_lb"], "init_strMap": sm,
           "iterations": np.int32(steps), "final_f": f, "final_u": u,
           "fma_spread_u": np.float64(rel(uf[m3], u[m3])), "fma_spread_f": np.float64(rel(ff[m19], f[m19]))}
    path = os.path.join(HERE, f"bgk_{name}.npz")
    np.savez_compressed(path, **out)
    return os.path.getsize(path)


if __name__ == "__main__":
    if not po.srt_available():
        sys.exit("oracle/_ref/srt_driver is not built: run oracle/refbuild/build_ref.sh first")
    for nm, n in BGK_CASES.items():
        print(f"bgk_{nm}: {make(nm, n) / 1024:.1f} KiB")
