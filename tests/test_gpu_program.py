"""The simulation program (bin/d3q19_b200, the drop-in for the reference's
executable) run on the reference's own input files: with the reference's
arithmetic its output files are byte-identical to the reference's; with the
fast arithmetic every printed number agrees to the printed precision up to
a few units in the last digit."""
import os
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import GOLDEN, PKG, load_golden
from cases import CASES, input_keywords, is_variable

import d3q19_b200 as d3

pytestmark = pytest.mark.gpu

FILES = ["velocity_field_final.txt", "matlab_postproc/velocity_field_centerline.txt", "velocity_profile_z.txt",
         "xyz_ovito_output.txt"]


def run_program(name, **extra):
    extra.setdefault("use_constant_viscosity", 0 if is_variable(CASES[name]) else 1)
    d = tempfile.mkdtemp(prefix="d3q19prog_")
    os.makedirs(os.path.join(d, "matlab_postproc"))
    os.makedirs(os.path.join(d, "unit_sphere_partitions"))
    with np.load(os.path.join(GOLDEN, "unit_sphere_partitions.npz")) as z:
        for k in z.files:
            with open(os.path.join(d, "unit_sphere_partitions", f"unit_sphere_partition_{k[1:]}.txt"), "wb") as fh:
                fh.write(z[k].tobytes())
    kw = dict(input_keywords(CASES[name]), **extra)
    with open(os.path.join(d, "input_file.txt"), "w") as fh:
        fh.write(d3.keywords_text(kw))
    p = subprocess.run([os.path.join(PKG, "bin", "d3q19_b200")], cwd=d, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
    return d, p.stdout


@pytest.mark.parametrize("name", ["couette", "sphere_wrap", "contacts", "casson"])
def test_program_outputs_identical_to_reference(name):
    g = load_golden(name)
    d, out = run_program(name, reference_arithmetic=1)
    for fn in FILES:
        key = "file_" + fn.replace("/", "__")
        if key in g:
            assert open(os.path.join(d, fn), "rb").read() == g[key].tobytes(), fn
    if CASES[name].get("num_particles", 0):
        ref_tail = g["stdout_tail"].tobytes().decode()
        want = [ln for ln in ref_tail.split("\n") if ln.startswith("Final force on particle 1")]
        got = [ln for ln in out.split("\n") if ln.startswith("Final force on particle 1")]
        assert want and got == want
    shutil.rmtree(d)


def _numbers(text):
    return np.array([float(w) for w in text.replace(",", " ").split() if _isnum(w)])


def _isnum(w):
    try:
        float(w)
        return True
    except ValueError:
        return False


@pytest.mark.parametrize("name", ["couette", "sphere_wrap"])
def test_program_outputs_fast_arithmetic(name):
    """Fast arithmetic: same files, same layout, every printed number within
    a few units of its last printed digit (%9.7f / %f)."""
    g = load_golden(name)
    d, _ = run_program(name)
    for fn in FILES:
        key = "file_" + fn.replace("/", "__")
        if key not in g:
            continue
        a = _numbers(open(os.path.join(d, fn)).read())
        b = _numbers(g[key].tobytes().decode())
        assert a.shape == b.shape, fn
        assert np.abs(a - b).max() <= 5e-6, fn
    shutil.rmtree(d)


def test_program_stops_on_a_malformed_sphere_file():
    # Exit status 1 and the reference's message, before the device is used
    # for the run (the reference exits in the same place).
    d = tempfile.mkdtemp(prefix="d3q19prog_")
    os.makedirs(os.path.join(d, "matlab_postproc"))
    os.makedirs(os.path.join(d, "unit_sphere_partitions"))
    with open(os.path.join(d, "unit_sphere_partitions", "unit_sphere_partition_256.txt"), "w") as fh:
        fh.write("0,0,1\n" * 40)  # truncated
    kw = dict(iterations=5, total_lattice_size=(24, 24, 24), boundary_conditions_xyz=(0, 0, 1), num_particles=1,
              particle_diameter=8.0, initial_particle_distribution=3, initial_particle_buffer=11.0,
              domain_decomposition=(1, 1, 1))
    with open(os.path.join(d, "input_file.txt"), "w") as fh:
        fh.write(d3.keywords_text(kw))
    p = subprocess.run([os.path.join(PKG, "bin", "d3q19_b200")], cwd=d, capture_output=True, text=True, timeout=120)
    assert p.returncode == 1 and "malformed coordinates read in sphere discretization" in p.stderr
    assert not os.path.exists(os.path.join(d, "velocity_field_final.txt"))
