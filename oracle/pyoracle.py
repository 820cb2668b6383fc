"""ctypes wrapper around the oracle restatement (oracle/d3q19_oracle.c) and a
runner for the reference itself built by oracle/refbuild/build_ref.sh.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline / reference legs of bench.py, never by the product package.
"""
from __future__ import annotations

import ctypes as C
import os
import shutil
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(BUILD, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

INT_FIELDS = [
    ("MaxIterations", 1), ("BasisVel", 57), ("LatticeSize", 3), ("SystemSize", 3), ("BufferSize", 3),
    ("BoundaryConds", 3), ("NumZones", 3), ("MaintainShear", 1), ("ViscosityModel", 1), ("NumParticles", 1),
    ("ParForceModel", 1), ("MaxSurfPointsPerNode", 1), ("InterpOrderIBM", 1), ("PointsPerParticle", 1),
    ("PointsPerWorkGroup", 1), ("TotalSurfPoints", 1), ("WorkGroupsPerParticle", 1)]
FLP_FIELDS = [
    ("ConstBodyForce", 3), ("EqWeights", 19), ("VelUpper", 3), ("VelLower", 3), ("NewtonianTau", 1),
    ("ViscosityParams", 4), ("ZoneWidth", 3), ("ParticleDiam", 1), ("ParticleMass", 1), ("PointArea", 1),
    ("ParticleMomInertia", 1), ("ParForceParams", 2), ("ParticleZBuffer", 1), ("DirectForcingCoeff", 1)]


def _struct(fields, ctype):
    class S(C.Structure):
        _fields_ = [(n, ctype * k) if k > 1 else (n, ctype) for n, k in fields]
    return S


IntParams = _struct(INT_FIELDS, C.c_int)
FlpParams = _struct(FLP_FIELDS, C.c_float)
assert C.sizeof(IntParams) == 332 and C.sizeof(FlpParams) == 176


def build(force: bool = False) -> str:
    """Compile the oracle restatement into oracle/_build/liboracle.so."""
    os.makedirs(BUILD, exist_ok=True)
    src = os.path.join(HERE, "d3q19_oracle.c")
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        subprocess.check_call(["gcc", "-O2", "-ffp-contract=off", "-fopenmp", "-fPIC", "-shared", "-std=gnu11",
                               src, "-o", LIB, "-lm"])
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        _lib = C.CDLL(LIB)
        _lib.orc_create_periodic_stream_mapping.restype = C.c_int
        _lib.orc_tau_clamp_count.restype = C.c_longlong
    return _lib


def params_from_bytes(ib: bytes, fb: bytes):
    ip = IntParams.from_buffer_copy(ib)
    fp = FlpParams.from_buffer_copy(fb)
    return ip, fp


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


class OracleState:
    """Holds the reference's buffers (numpy arrays in the reference layouts)
    and advances them with the oracle's restatement of sim_main.c:324-447."""

    def __init__(self, ip, fp, arrays: dict, num_par_threads: int, rebuild_freq: int,
                 variable_viscosity: bool, tangential=(0, 0, 0)):
        self.ip, self.fp = ip, fp
        self.a = {k: np.ascontiguousarray(v).copy() for k, v in arrays.items()}
        self.num_par_threads = num_par_threads
        self.rebuild_freq = rebuild_freq
        self.variable = int(variable_viscosity)
        self.tangential = tangential

    def _cstate(self):
        a = self.a
        fields = [("fA", "fA"), ("fB", "fB"), ("u", "u"), ("gpf", "gpf"), ("tau_lb", "tau_lb"),
                  ("countPoint", "countPoint"), ("parKin", "parKin"), ("parForce", "parForce"),
                  ("parFluidForce", "parFluidForce"), ("spherePoints", "spherePoints"), ("strMap", "strMap")]

        class S(C.Structure):
            _fields_ = [("fA", C.c_void_p), ("fB", C.c_void_p), ("u", C.c_void_p), ("gpf", C.c_void_p),
                        ("tau_lb", C.c_void_p), ("countPoint", C.c_void_p), ("parKin", C.c_void_p),
                        ("parForce", C.c_void_p), ("parFluidForce", C.c_void_p), ("spherePoints", C.c_void_p),
                        ("strMap", C.c_void_p), ("numPeriodicNodes", C.c_int), ("zoneNeighDat", C.c_void_p),
                        ("parsZone", C.c_void_p), ("zoneMembers", C.c_void_p), ("numParInZone", C.c_void_p),
                        ("threadMembers", C.c_void_p), ("numParInThread", C.c_void_p),
                        ("numParThreads", C.c_int), ("rebuildFreq", C.c_int), ("variable_viscosity", C.c_int),
                        ("tangentialVelBC", C.c_int * 3)]
        s = S()
        for f, k in fields:
            setattr(s, f, _p(a.get(k)))
        s.numPeriodicNodes = len(a["strMap"]) // 2
        for k in ("zoneNeighDat", "parsZone", "zoneMembers", "numParInZone", "threadMembers", "numParInThread"):
            setattr(s, k, _p(a.get(k)))
        s.numParThreads = self.num_par_threads
        s.rebuildFreq = self.rebuild_freq
        s.variable_viscosity = self.variable
        s.tangentialVelBC = (C.c_int * 3)(*self.tangential)
        return s

    def step(self, t: int):
        s = self._cstate()
        lib().orc_step(C.byref(s), C.byref(self.ip), C.byref(self.fp), C.c_int(t))

    def run(self, t0: int, n: int):
        for t in range(t0, t0 + n):
            self.step(t)

    def latest_f(self, t_last: int):
        """Distribution buffer written by step t_last (sim_main.c:324-337)."""
        return self.a["fA"] if t_last % 2 == 1 else self.a["fB"]


# --- the reference itself (oracle/_ref), run through the mock runtime ----------

# Creation order of the reference's buffers, sim_main.c:121-190 (the mock
# runtime numbers dumps by creation order).
REF_BUFFERS = ["fA", "fB", "u", "gpf", "countPoint", "tau_lb", "parKin", "parForce", "parFluidForce", "parsZone",
               "zoneMembers", "numParInZone", "parFluidForceSum", "threadMembers", "numParInThread", "zoneNeighDat",
               "intDat", "flpDat", "strMap", "spherePoints"]
_INT_BUFS = {"countPoint", "parsZone", "zoneMembers", "numParInZone", "threadMembers", "numParInThread",
             "zoneNeighDat", "strMap"}


def ref_available() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "ref_const")) and os.path.isdir(os.path.join(REF_DIR, "run_data"))


def write_input_file(path: str, keywords: dict):
    with open(path, "w") as fh:
        for k, v in keywords.items():
            if isinstance(v, (list, tuple)):
                v = " ".join(str(x) for x in v)
            fh.write(f"{k:<32s}{v}\n")


def run_reference(keywords: dict, variable_viscosity: bool = False, serial: bool = True, dump: bool = True,
                  threads: int | None = None, workdir: str | None = None, timeout: float = 3600.0,
                  extra_env: dict | None = None):
    """Run the reference binary on an input-file keyword dict in a scratch
    directory.  Returns (stdout, {buffer name: bytes}, workdir)."""
    exe = os.path.join(REF_DIR, "ref_var" if variable_viscosity else "ref_const")
    wd = workdir or tempfile.mkdtemp(prefix="d3q19ref_")
    os.makedirs(os.path.join(wd, "matlab_postproc"), exist_ok=True)
    data = os.path.join(REF_DIR, "run_data")
    for f in ("GPU_program.cl", "CPU_program.cl"):
        shutil.copy(os.path.join(data, f), os.path.join(wd, f))
    usp = os.path.join(wd, "unit_sphere_partitions")
    if not os.path.exists(usp):
        shutil.copytree(os.path.join(data, "unit_sphere_partitions"), usp)
    write_input_file(os.path.join(wd, "input_file.txt"), keywords)
    env = dict(os.environ)
    env["MOCKCL_QUIET"] = "1"
    if serial:
        env["MOCKCL_SERIAL"] = "1"
    if threads:
        env["MOCKCL_THREADS"] = str(threads)
    dd = os.path.join(wd, "dump")
    if dump:
        os.makedirs(dd, exist_ok=True)
        env["MOCKCL_DUMP_DIR"] = dd
    if extra_env:
        env.update(extra_env)
    p = subprocess.run([exe], cwd=wd, env=env, capture_output=True, text=True, timeout=timeout)
    if p.returncode != 0:
        raise RuntimeError(f"reference run failed ({p.returncode}):\n{p.stdout[-2000:]}\n{p.stderr[-2000:]}")
    bufs = {}
    if dump:
        for i, name in enumerate(REF_BUFFERS):
            fn = os.path.join(dd, f"buf_{i:02d}.bin")
            if os.path.exists(fn):
                with open(fn, "rb") as fh:
                    bufs[name] = fh.read()
    return p.stdout, bufs, wd


def ref_arrays(bufs: dict) -> dict:
    out = {}
    for k, b in bufs.items():
        if k in ("intDat", "flpDat"):
            out[k] = np.frombuffer(b, dtype=np.uint8).copy()
        elif k in _INT_BUFS:
            out[k] = np.frombuffer(b, dtype=np.int32).copy()
        else:
            out[k] = np.frombuffer(b, dtype=np.float32).copy()
    return out


def srt_available() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "srt_driver"))


def run_srt(int_bytes: bytes, flp_bytes: bytes, f, g, strMap, nsteps: int, timeout: float = 600.0, fma=False):
    """The reference's BGK kernel collideSRT_newtonian_stream_D3Q19 with its
    periodic and velocity boundary kernels, nsteps steps in the host's order
    (oracle/refbuild/srt_driver.c), from distributions f (19*N_C), body-force
    field g (3*N_C) and the periodic node list strMap.  Returns (f, u) after
    the last step (post-boundary f).  fma: the kernels compiled with fused
    multiply-add contraction (srt_driver_fma)."""
    ip = IntParams.from_buffer_copy(int_bytes)
    nc = ip.LatticeSize[0] * ip.LatticeSize[1] * ip.LatticeSize[2]
    strMap = np.ascontiguousarray(strMap, np.int32)
    with tempfile.TemporaryDirectory(prefix="d3q19srt_") as wd:
        src, dst = os.path.join(wd, "in.bin"), os.path.join(wd, "out.bin")
        with open(src, "wb") as fh:
            fh.write(int_bytes)
            fh.write(flp_bytes)
            fh.write(np.array([nsteps, strMap.size // 2], np.int32).tobytes())
            fh.write(np.ascontiguousarray(f, np.float32).tobytes())
            fh.write(np.ascontiguousarray(g, np.float32).tobytes())
            fh.write(strMap.tobytes())
        shutil.copy(os.path.join(REF_DIR, "run_data", "GPU_program.cl"), os.path.join(wd, "GPU_program.cl"))
        env = dict(os.environ, MOCKCL_QUIET="1")
        exe = os.path.join(REF_DIR, "srt_driver_fma" if fma else "srt_driver")
        p = subprocess.run([exe, src, dst], cwd=wd, env=env, capture_output=True,
                           text=True, timeout=timeout)
        if p.returncode != 0:
            raise RuntimeError(f"srt_driver failed ({p.returncode}): {p.stderr[-2000:]}")
        out = np.fromfile(dst, np.float32)
    return out[: 19 * nc].copy(), out[19 * nc:].copy()
