"""The bounds-checked build (lib/libd3q19_b200_checked.so, -DD3Q19_BOUNDS_CHECK=1).

Its kernels check the data-dependent device indices (pull sources, marker
ids read from the tile lists, interpolation stencils, zone and sphere ids of
the contact search) and report D3Q19_EBOUNDS instead of touching memory
outside an array.  Here it runs in a child process (the build is chosen when
the library is first loaded) on cases that exercise periodic wrap, wrapping
sphere stencils, tile-edge markers, contacts and the batched pool, each with
two distribution buffers and in place (the in-place odd step pulls from
upwind and pushes downwind, so its indices are checked too).  It must
report nothing, and its results must be bit-identical to the default
build's, since the checks change no arithmetic.
"""
import os
import subprocess
import sys
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
CASE_NAMES = ["sphere_wrap", "wrap_tile_edge", "contacts", "power_law_sphere", "periodic_force"]
INPLACE_NAMES = ["sphere_wrap", "wrap_tile_edge", "contacts", "couette", "xwall_tangential"]


def compute(out_path):
    """Runs every case with the library this process loaded; saves the
    results to out_path."""
    import d3q19_b200 as d3
    from conftest import load_golden
    from cases import CASES
    from gpu_helpers import sim_from_golden
    from d3q19_b200 import serving as sv

    res = {}
    runs = [(n, 0) for n in CASE_NAMES] + [(n, 1) for n in INPLACE_NAMES]
    for name, inplace in runs:
        g = load_golden(name)
        sim, ip, fp = sim_from_golden(g, CASES[name], inplace=inplace)
        sim.run(1, 3 * CASES[name]["iterations"] + inplace)  # in place: end on an odd step
        sim.synchronize()
        key = f"{name}/ip{inplace}"
        res[f"{key}/u"] = sim.read_u()
        res[f"{key}/f"] = sim.read_f()
        if sim.np > 0:
            res[f"{key}/kin"] = sim.read_parkin()
            res[f"{key}/pff"] = sim.read_parfluidforce()
            res[f"{key}/gpf"] = sim.read_spread_force()
        sim.close()
    reqs = [sv.ShearRequest(rid=0, edge=(34, 34, 34), phi=0.25, model="power_law", wall_speed=0.03, seed=5),
            sv.ShearRequest(rid=1, edge=(32, 40, 36), phi=0.2, model="casson", wall_speed=0.02, seed=6)]
    for inplace in (False, True):
        pool = d3.Pool(storage=1, max_slots=4, inplace=inplace)
        slots = [pool.admit(sv.host_state(r)) for r in reqs]
        pool.advance(110)
        st, _, _, code = pool.mean_stress_all(4)
        for k, s in enumerate(slots):
            assert code[s] == 0, (k, inplace, d3.STATUS[int(code[s])])
            res[f"pool{k}/ip{int(inplace)}/u"] = pool.member(s).read_u()
        pool.close()
    np.savez(out_path, **res)


def test_checked_build_reports_nothing_and_matches():
    import d3q19_b200 as d3

    checked = os.path.join(os.path.dirname(d3.CUDA_LIB), "libd3q19_b200_checked.so")
    assert os.path.exists(checked), "build the checked library (build.py)"
    d = tempfile.mkdtemp(prefix="d3q19bc_")
    env = dict(os.environ, D3Q19_BOUNDS_CHECK="1")
    p = subprocess.run([sys.executable, os.path.abspath(__file__), os.path.join(d, "checked.npz")], env=env,
                       capture_output=True, text=True, timeout=600, cwd=os.path.dirname(HERE))
    assert p.returncode == 0, p.stdout[-3000:] + p.stderr[-3000:]
    compute(os.path.join(d, "default.npz"))
    with np.load(os.path.join(d, "checked.npz")) as a, np.load(os.path.join(d, "default.npz")) as b:
        assert sorted(a.files) == sorted(b.files)
        for k in a.files:
            assert np.array_equal(a[k].view(np.uint8), b[k].view(np.uint8)), k


if __name__ == "__main__":
    sys.path[:0] = [HERE, os.path.join(HERE, "golden"), os.path.join(os.path.dirname(HERE),
                                                                     "dispersion-shear_d3q19-opencl_b200")]
    import d3q19_b200 as d3

    assert d3.CUDA_LIB.endswith("_checked.so"), d3.CUDA_LIB
    compute(sys.argv[1])
