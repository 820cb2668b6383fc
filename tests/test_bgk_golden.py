"""The BGK golden vectors (tests/golden/bgk_<case>.npz) are the reference's own
BGK kernel collideSRT_newtonian_stream_D3Q19 (GPU_program.cl:868-947) with its
boundary kernels in the host's step order (oracle/refbuild/srt_driver.c): a
re-run through oracle/_ref reproduces them bit for bit."""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def load(name):
    with np.load(os.path.join(HERE, "golden", f"bgk_{name}.npz")) as z:
        return {k: z[k] for k in z.files}


@pytest.mark.parametrize("name", ["couette", "periodic_force"])
def test_fixture_is_the_reference_srt_kernel(name):
    from oracle import pyoracle as po

    if not po.srt_available():
        pytest.skip("oracle/_ref/srt_driver (the reference built for the host) is not present")
    import sys

    sys.path.insert(0, os.path.join(HERE, "golden"))
    from make_golden_bgk import srt_inputs

    g = load(name)
    ib, fb, f0, force, sm = srt_inputs(g)
    f, u = po.run_srt(ib, fb, f0, force, sm, int(g["iterations"]))
    assert np.array_equal(f.view(np.uint32), g["final_f"].view(np.uint32))
    assert np.array_equal(u.view(np.uint32), g["final_u"].view(np.uint32))
