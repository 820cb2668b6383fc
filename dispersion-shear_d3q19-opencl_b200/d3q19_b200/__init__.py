"""Python binding of the B200 D3Q19 LBM + IBM library (ctypes over the C ABI
of include/d3q19_b200.h and the C host routines of host/d3q19_host.h).

The GPU path runs only through lib/libd3q19_b200.so; if that library (or a
usable sm_100 device) is missing, the calls raise -- there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np

PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(PKG, "lib")
# D3Q19_BOUNDS_CHECK=1 in the environment selects the bounds-checked build
# (device index checks that report D3Q19_EBOUNDS instead of faulting).
CUDA_LIB = os.path.join(LIBDIR, "libd3q19_b200_checked.so" if os.environ.get("D3Q19_BOUNDS_CHECK") == "1"
                        else "libd3q19_b200.so")
HOST_LIB = os.path.join(LIBDIR, "libd3q19_host.so")

# Largest lattice (N_C nodes) d3q19_read_spread_force_static accepts.
STATIC_SPREAD_MAX_CELLS = 262144
STATUS = {0: "OK", -1: "EINVAL", -2: "ENOMEM", -3: "ECUDA", -4: "ENODEV", -5: "EOVERFLOW", -6: "ENUMERIC",
          -7: "ESTATE", -8: "EBUSY", -9: "EBOUNDS", -10: "ETIMEDOUT"}
EBUSY = -8

_INT_FIELDS = [
    ("MaxIterations", 1), ("BasisVel", 57), ("LatticeSize", 3), ("SystemSize", 3), ("BufferSize", 3),
    ("BoundaryConds", 3), ("NumZones", 3), ("MaintainShear", 1), ("ViscosityModel", 1), ("NumParticles", 1),
    ("ParForceModel", 1), ("MaxSurfPointsPerNode", 1), ("InterpOrderIBM", 1), ("PointsPerParticle", 1),
    ("PointsPerWorkGroup", 1), ("TotalSurfPoints", 1), ("WorkGroupsPerParticle", 1)]
_FLP_FIELDS = [
    ("ConstBodyForce", 3), ("EqWeights", 19), ("VelUpper", 3), ("VelLower", 3), ("NewtonianTau", 1),
    ("ViscosityParams", 4), ("ZoneWidth", 3), ("ParticleDiam", 1), ("ParticleMass", 1), ("PointArea", 1),
    ("ParticleMomInertia", 1), ("ParForceParams", 2), ("ParticleZBuffer", 1), ("DirectForcingCoeff", 1)]


def _fields(spec, ct):
    return [(n, ct * k) if k > 1 else (n, ct) for n, k in spec]


class IntParams(C.Structure):
    """int_param_struct (struct_header_device.h:4-31)."""
    _fields_ = _fields(_INT_FIELDS, C.c_int)


class FlpParams(C.Structure):
    """flp_param_struct (struct_header_device.h:34-57)."""
    _fields_ = _fields(_FLP_FIELDS, C.c_float)


class Options(C.Structure):
    _fields_ = [("variable_viscosity", C.c_int), ("collision", C.c_int), ("storage", C.c_int),
                ("particle_precision", C.c_int), ("fixed_particles", C.c_int), ("num_par_threads", C.c_int),
                ("rebuild_freq", C.c_int), ("tangential_vel_bc", C.c_int * 3), ("tau_max", C.c_float),
                ("tau_min", C.c_float), ("casson_reg", C.c_float), ("device", C.c_int),
                ("ibm_tile_capacity", C.c_int), ("arithmetic", C.c_int), ("inplace", C.c_int),
                ("fluid_kernel", C.c_int), ("periodic_smoothing", C.c_int)]


class DeviceInfo(C.Structure):
    _fields_ = [("name", C.c_char * 256), ("sm_count", C.c_int), ("cc_major", C.c_int), ("cc_minor", C.c_int),
                ("global_mem_bytes", C.c_size_t), ("kernel_work_group_size", C.c_int)]


class HostParams(C.Structure):
    _fields_ = [("ConsolePrintFreq", C.c_int), ("InitialDist", C.c_char * 128), ("InitialVel", C.c_float * 3),
                ("InitialParticleDistribution", C.c_int), ("ParticleBuffer", C.c_float),
                ("InterpOrderIBM", C.c_int), ("DomainDecomp", C.c_int * 3), ("ParticleDensity", C.c_float),
                ("RebuildFreq", C.c_int), ("VideoFreq", C.c_int), ("FluidOutputSpacing", C.c_int),
                ("TangentialVelBC", C.c_int * 3), ("ShearStressFreq", C.c_int), ("RandParticleShift", C.c_float),
                ("UseConstantViscosity", C.c_int), ("PointsOverride", C.c_int), ("FixedParticles", C.c_int),
                ("ParticleSeed", C.c_uint), ("MinParticleGap", C.c_float), ("TauMax", C.c_float),
                ("TauMin", C.c_float), ("CassonReg", C.c_float), ("Collision", C.c_int), ("Storage", C.c_int),
                ("ParticlePrecision", C.c_int), ("Arithmetic", C.c_int), ("Fp64Build", C.c_int),
                ("Inplace", C.c_int), ("PeriodicSmoothing", C.c_int)]


class Config(C.Structure):
    """d3q19h_config: the reference's two parameter blocks + host parameters."""
    _fields_ = [("ip", IntParams), ("fp", FlpParams), ("hp", HostParams)]


assert C.sizeof(IntParams) == 332 and C.sizeof(FlpParams) == 176

_cuda = None
_host = None


class D3Q19Error(RuntimeError):
    pass


def cuda_lib():
    """The CUDA library; raises when it is missing (no fallback)."""
    global _cuda
    if _cuda is None:
        if not os.path.exists(CUDA_LIB):
            raise D3Q19Error(f"{CUDA_LIB} is not built (run build.py); there is no CPU path")
        lib = C.CDLL(CUDA_LIB)
        P = C.c_void_p
        lib.d3q19_create.argtypes = [C.POINTER(IntParams), C.POINTER(FlpParams), C.POINTER(Options),
                                     C.POINTER(C.c_void_p)]
        lib.d3q19_last_error.restype = C.c_char_p
        lib.d3q19_last_error.argtypes = [P]
        lib.d3q19_tau_clamp_count.restype = C.c_longlong
        lib.d3q19_tau_clamp_count.argtypes = [P]
        lib.d3q19_stream.restype = P
        lib.d3q19_stream.argtypes = [P]
        lib.d3q19_periodic_map.argtypes = [C.POINTER(IntParams), P, C.c_int]
        for name in ("d3q19_write_lattice", "d3q19_write_particles", "d3q19_write_zones", "d3q19_read_u",
                     "d3q19_read_tau", "d3q19_read_parkin", "d3q19_read_parforce", "d3q19_read_parfluidforce",
                     "d3q19_read_f", "d3q19_read_spread_force", "d3q19_read_spread_force_static",
                     "d3q19_read_marker_cells", "d3q19_read_zones", "d3q19_plane_stats", "d3q19_shear_profile",
                     "d3q19_mean_stress",
                     "d3q19_synchronize", "d3q19_destroy", "d3q19_write_periodic_map"):
            getattr(lib, name).restype = C.c_int
        lib.d3q19_step.argtypes = [P, C.c_int]
        lib.d3q19_profile.argtypes = [P, C.c_int]
        lib.d3q19_profile_read.argtypes = [P, C.POINTER(C.c_double), C.POINTER(C.c_int), C.POINTER(C.c_double),
                                           C.POINTER(C.c_int)]
        lib.d3q19_run.argtypes = [P, C.c_int, C.c_int]
        for name in ("d3q19_k_collide_stream", "d3q19_k_particles", "d3q19_k_contacts"):
            getattr(lib, name).argtypes = [P, C.c_int]
        lib.d3q19_k_zones.argtypes = [P]
        lib.d3q19_write_periodic_map.argtypes = [P, P, C.c_int]
        lib.d3q19_read_parkin64.restype = C.c_int
        lib.d3q19_context_bytes.argtypes = [C.POINTER(IntParams), C.POINTER(Options), C.POINTER(C.c_size_t)]
        lib.d3q19_pool_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_size_t, C.POINTER(C.c_void_p)]
        lib.d3q19_pool_admit.argtypes = [P, C.POINTER(IntParams), C.POINTER(FlpParams), C.POINTER(Options)] + \
            [P] * 11 + [C.POINTER(C.c_int)]
        lib.d3q19_pool_advance.argtypes = [P, C.c_int]
        lib.d3q19_pool_context.restype = P
        lib.d3q19_pool_context.argtypes = [P, C.c_int]
        lib.d3q19_pool_slot_steps.restype = C.c_longlong
        lib.d3q19_pool_slot_steps.argtypes = [P, C.c_int]
        lib.d3q19_pool_release.argtypes = [P, C.c_int]
        lib.d3q19_pool_usage.argtypes = [P, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t), C.POINTER(C.c_int)]
        lib.d3q19_pool_set_grid.argtypes = [P, C.c_int, C.c_int, C.c_int]
        lib.d3q19_pool_get_grid.argtypes = [P, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
        lib.d3q19_pool_autotune.argtypes = [P, C.c_int]
        lib.d3q19_pool_tune_state.argtypes = [P] + [C.POINTER(C.c_int)] * 5
        lib.d3q19_pool_tune_trials.argtypes = [P, P, P, P, C.c_int, C.POINTER(C.c_int)]
        lib.d3q19_tune_export.argtypes = [C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]
        lib.d3q19_tune_import.argtypes = [C.c_char_p]
        lib.d3q19_tune_clear.argtypes = []
        lib.d3q19_pool_synchronize.argtypes = [P]
        lib.d3q19_pool_poll.argtypes = [P]
        lib.d3q19_pool_stream.restype = P
        lib.d3q19_pool_stream.argtypes = [P]
        lib.d3q19_pool_last_error.restype = C.c_char_p
        lib.d3q19_pool_last_error.argtypes = [P]
        lib.d3q19_pool_destroy.argtypes = [P]
        lib.d3q19_pool_mean_stress.argtypes = [P, P, P, P, P]
        lib.d3q19_checkpoint_bytes.argtypes = [P, C.POINTER(C.c_size_t)]
        lib.d3q19_checkpoint.argtypes = [P, P, C.c_size_t]
        lib.d3q19_restore.argtypes = [P, P, C.c_size_t]
        lib.d3q19_pool_evict.argtypes = [P, C.c_int, P, C.c_size_t]
        lib.d3q19_pool_readmit.argtypes = [P, C.POINTER(IntParams), C.POINTER(FlpParams), C.POINTER(Options), P,
                                           C.c_size_t, C.POINTER(C.c_int)]
        _cuda = lib
    return _cuda


def host_lib():
    global _host
    if _host is None:
        if not os.path.exists(HOST_LIB):
            raise D3Q19Error(f"{HOST_LIB} is not built (run build.py)")
        lib = C.CDLL(HOST_LIB)
        lib.d3q19h_parse_text.argtypes = [C.c_char_p, C.POINTER(Config)]
        lib.d3q19h_sphere_discretization.argtypes = [C.POINTER(Config), C.c_char_p, C.POINTER(C.POINTER(C.c_float))]
        lib.d3q19h_eqsp_points.argtypes = [C.c_int, C.c_void_p]
        lib.d3q19h_work_groups.argtypes = [C.POINTER(Config), C.c_int]
        lib.d3q19h_init_lattice.argtypes = [C.POINTER(Config), C.c_void_p, C.c_void_p, C.c_void_p]
        lib.d3q19h_init_particles.argtypes = [C.POINTER(Config), C.c_void_p, C.c_void_p, C.c_void_p]
        lib.d3q19h_zone_grid.argtypes = [C.POINTER(Config)]
        lib.d3q19h_zone_count.argtypes = [C.POINTER(Config)]
        lib.d3q19h_init_zones.argtypes = [C.POINTER(Config)] + [C.c_void_p] * 7
        lib.d3q19h_options.argtypes = [C.POINTER(Config), C.POINTER(Options)]
        lib.d3q19h_compute_shear_stress.argtypes = [C.c_void_p, C.POINTER(Config), C.c_void_p, C.c_char_p]
        lib.d3q19h_write_lattice_field.argtypes = [C.POINTER(Config), C.c_void_p, C.c_char_p, C.c_char_p]
        lib.d3q19h_check.argtypes = [C.POINTER(Config)]
        _host = lib
    return _host


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _fmt(v):
    if isinstance(v, (list, tuple)):
        return " ".join(str(x) for x in v)
    return str(v)


def keywords_text(keywords: dict) -> str:
    return "".join(f"{k:<32s}{_fmt(v)}\n" for k, v in keywords.items())


def parse_config(text: str) -> Config:
    cfg = Config()
    host_lib().d3q19h_parse_text(text.encode(), C.byref(cfg))
    return cfg


def device_info(device: int = 0) -> DeviceInfo:
    di = DeviceInfo()
    rc = cuda_lib().d3q19_get_device_info(device, C.byref(di))
    if rc:
        raise D3Q19Error(f"d3q19_get_device_info: {STATUS.get(rc, rc)}: {cuda_lib().d3q19_last_error(None)!r}")
    return di


def periodic_map(ip: IntParams) -> np.ndarray:
    lib = cuda_lib()
    n = lib.d3q19_periodic_map(C.byref(ip), None, 0)
    out = np.zeros(2 * max(n, 1), np.int32)
    lib.d3q19_periodic_map(C.byref(ip), _ptr(out), out.size)
    return out[: 2 * n]


def eqsp_points(n: int) -> np.ndarray:
    out = np.zeros(3 * n, np.float64)
    host_lib().d3q19h_eqsp_points(n, _ptr(out))
    return out.reshape(n, 3)


class HostState:
    """The initial state the reference's host builds (D3Q19-OpenCL.c host
    routines, in sim_main.c's order), computed by the C host library."""

    def __init__(self, cfg: Config, data_dir: str = ".", kernel_work_group_size: int = 256):
        h = host_lib()
        self.cfg = cfg
        if h.d3q19h_check(C.byref(cfg)):
            raise D3Q19Error("parameter check failed")
        pts = C.POINTER(C.c_float)()
        if h.d3q19h_sphere_discretization(C.byref(cfg), data_dir.encode(), C.byref(pts)) != 0:
            raise D3Q19Error("malformed sphere discretisation file")
        P = cfg.ip.PointsPerParticle
        self.spherePoints = np.ctypeslib.as_array(pts, shape=(4 * P,)).copy()
        C.CDLL(None).free(pts)
        h.d3q19h_work_groups(C.byref(cfg), kernel_work_group_size)
        ip = cfg.ip
        nc = ip.LatticeSize[0] * ip.LatticeSize[1] * ip.LatticeSize[2]
        self.f = np.zeros(19 * nc, np.float32)
        self.u = np.zeros(3 * nc, np.float32)
        self.tau = np.zeros(nc, np.float32)
        if h.d3q19h_init_lattice(C.byref(cfg), _ptr(self.f), _ptr(self.u), _ptr(self.tau)):
            raise D3Q19Error("lattice initialisation failed")
        np_ = ip.NumParticles
        nfa = max(ip.WorkGroupsPerParticle, 1)
        self.parKin = np.zeros(16 * max(np_, 2), np.float32)
        self.parForce = np.zeros(8 * max(np_, 1), np.float32)
        self.parFluidForce = np.zeros(8 * max(np_, 1) * nfa, np.float32)
        if h.d3q19h_init_particles(C.byref(cfg), _ptr(self.parKin), _ptr(self.parForce), _ptr(self.parFluidForce)):
            raise D3Q19Error("particle initialisation failed")
        self.parKin = self.parKin[: 16 * np_]
        self.parForce = self.parForce[: 8 * np_]
        self.parFluidForce = self.parFluidForce[: 8 * np_ * nfa]
        h.d3q19h_zone_grid(C.byref(cfg))
        Z = h.d3q19h_zone_count(C.byref(cfg))
        nth = cfg.hp.DomainDecomp[0] * cfg.hp.DomainDecomp[1] * cfg.hp.DomainDecomp[2]
        self.parsZone = np.zeros(max(np_, 1), np.int32)
        self.zoneMembers = np.zeros(Z * max(np_, 1), np.int32)
        self.numParInZone = np.zeros(Z, np.int32)
        self.threadMembers = np.zeros(max(nth, 1) * max(np_, 1), np.int32)
        self.numParInThread = np.zeros(max(nth, 1), np.int32)
        self.zoneNeighDat = np.zeros(28 * Z, np.int32)
        if np_ > 0 and h.d3q19h_init_zones(C.byref(cfg), _ptr(self.parKin), _ptr(self.parsZone),
                                           _ptr(self.zoneMembers), _ptr(self.numParInZone),
                                           _ptr(self.threadMembers), _ptr(self.numParInThread),
                                           _ptr(self.zoneNeighDat)):
            raise D3Q19Error("Particle out of bounds at zone initialization")
        self.options = Options()
        h.d3q19h_options(C.byref(cfg), C.byref(self.options))


class Simulation:
    """One GPU context: the reference's buffers resident on the device,
    advanced step by step in the reference's kernel order."""

    def __init__(self, ip: IntParams, fp: FlpParams, options: Options | None = None):
        self.lib = cuda_lib()
        self.ip = IntParams.from_buffer_copy(bytes(ip))
        self.fp = FlpParams.from_buffer_copy(bytes(fp))
        self.options = options or Options()
        h = C.c_void_p()
        rc = self.lib.d3q19_create(C.byref(self.ip), C.byref(self.fp), C.byref(self.options), C.byref(h))
        if rc:
            raise D3Q19Error(f"d3q19_create: {STATUS.get(rc, rc)}: {self.lib.d3q19_last_error(None).decode()}")
        self.h = h
        self.nc = self.ip.LatticeSize[0] * self.ip.LatticeSize[1] * self.ip.LatticeSize[2]
        self.np = self.ip.NumParticles
        self.nfa = max(self.ip.WorkGroupsPerParticle, 1)
        self.nzones = self.ip.NumZones[0] * self.ip.NumZones[1] * self.ip.NumZones[2]

    @classmethod
    def from_host_state(cls, hs: HostState, **option_overrides):
        opt = Options.from_buffer_copy(bytes(hs.options))
        for k, v in option_overrides.items():
            setattr(opt, k, v)
        sim = cls(hs.cfg.ip, hs.cfg.fp, opt)
        sim.write_lattice(hs.f, hs.u, hs.tau)
        sim.write_periodic_map(periodic_map(hs.cfg.ip))
        if sim.np > 0:
            sim.write_particles(hs.parKin, hs.parForce, hs.parFluidForce, hs.spherePoints)
            sim.write_zones(hs.zoneNeighDat, hs.parsZone, hs.zoneMembers, hs.numParInZone, hs.threadMembers,
                            hs.numParInThread)
        return sim

    def _check(self, rc, what):
        if rc:
            raise D3Q19Error(f"{what}: {STATUS.get(rc, rc)}: {self.lib.d3q19_last_error(self.h).decode()}")

    @property
    def fluid_kernel(self):
        """Collide-stream kernel of the context: 'tile' (fluid_step_kernel),
        'tma' (the TMA-pipelined fluid_tma_kernel) or 'reference-order'."""
        k = self.lib.d3q19_fluid_kernel(self.h)
        return {0: "tile", 1: "tma", 2: "reference-order"}[k]

    def write_lattice(self, f, u, tau=None):
        f = np.ascontiguousarray(f, np.float32)
        u = np.ascontiguousarray(u, np.float32)
        tau = None if tau is None else np.ascontiguousarray(tau, np.float32)
        self._check(self.lib.d3q19_write_lattice(self.h, _ptr(f), _ptr(u), _ptr(tau)), "write_lattice")

    def write_particles(self, parKin, parForce, parFluidForce, spherePoints):
        a = [np.ascontiguousarray(x, np.float32) for x in (parKin, parForce, parFluidForce, spherePoints)]
        self._check(self.lib.d3q19_write_particles(self.h, *[_ptr(x) for x in a]), "write_particles")

    def write_zones(self, znd, parsZone, zoneMembers, numParInZone, threadMembers=None, numParInThread=None):
        a = [None if x is None else np.ascontiguousarray(x, np.int32)
             for x in (znd, parsZone, zoneMembers, numParInZone, threadMembers, numParInThread)]
        self._check(self.lib.d3q19_write_zones(self.h, *[_ptr(x) for x in a]), "write_zones")

    def write_periodic_map(self, strMap):
        s = np.ascontiguousarray(strMap, np.int32)
        self._check(self.lib.d3q19_write_periodic_map(self.h, _ptr(s), len(s) // 2), "write_periodic_map")

    def step(self, t: int):
        self._check(self.lib.d3q19_step(self.h, t), "step")

    def step_by_pass(self, t: int, rebuild: bool):
        """Step t through the pass entry points (d3q19_k_*), in order."""
        self._check(self.lib.d3q19_k_collide_stream(self.h, t), "k_collide_stream")
        self._check(self.lib.d3q19_k_particles(self.h, t), "k_particles")
        self._check(self.lib.d3q19_k_contacts(self.h, t), "k_contacts")
        if rebuild:
            self._check(self.lib.d3q19_k_zones(self.h), "k_zones")

    def run(self, t0: int, n: int):
        self._check(self.lib.d3q19_run(self.h, t0, n), "run")

    def prepare_run(self, t0: int, n: int):
        """Captures the CUDA graphs run(t0, n) replays without running them
        (d3q19_prepare_run)."""
        self._check(self.lib.d3q19_prepare_run(self.h, t0, n), "prepare_run")

    def synchronize(self):
        self._check(self.lib.d3q19_synchronize(self.h), "synchronize")

    def _read(self, fn, n, dtype=np.float32, out=None):
        """out: an existing C-contiguous array of n elements of dtype to read
        into (for example pinned host memory), else a new one."""
        if out is None:
            out = np.zeros(n, dtype)
        elif out.dtype != dtype or out.size != n or not out.flags.c_contiguous:
            raise ValueError(f"{fn}: out must be a contiguous {dtype.__name__} array of {n} elements")
        self._check(getattr(self.lib, fn)(self.h, _ptr(out)), fn)
        return out

    def read_u(self, out=None):
        return self._read("d3q19_read_u", 3 * self.nc, out=out)

    def read_tau(self):
        return self._read("d3q19_read_tau", self.nc)

    def read_f(self):
        return self._read("d3q19_read_f", 19 * self.nc)

    def read_parkin(self, out=None):
        return self._read("d3q19_read_parkin", 16 * self.np, out=out)

    def read_parkin64(self):
        """The FP64 sphere state (particle_precision = 1 or the FP64 build)."""
        return self._read("d3q19_read_parkin64", 16 * self.np, np.float64)

    def read_parforce(self):
        return self._read("d3q19_read_parforce", 8 * self.np)

    def read_parfluidforce(self, out=None):
        return self._read("d3q19_read_parfluidforce", 8 * self.np * self.nfa, out=out)

    def read_spread_force(self):
        return self._read("d3q19_read_spread_force", 3 * self.nc)

    def read_spread_force_static(self):
        """The spread force field through the entry point that allocates no
        device memory (lattices of up to STATIC_SPREAD_MAX_CELLS nodes)."""
        return self._read("d3q19_read_spread_force_static", 3 * self.nc)

    def read_marker_cells(self):
        return self._read("d3q19_read_marker_cells", 3 * self.np * self.ip.PointsPerParticle, np.int32)

    def read_zones(self):
        pz = np.zeros(self.np, np.int32)
        zm = np.zeros(self.nzones * self.np, np.int32)
        nz = np.zeros(self.nzones, np.int32)
        self._check(self.lib.d3q19_read_zones(self.h, _ptr(pz), _ptr(zm), _ptr(nz)), "read_zones")
        return pz, zm, nz

    def plane_stats(self):
        """Per-plane FP64 sums, shape (Nz, 5): u_x, u_y, u_z, shear rate,
        viscous shear stress (d3q19_plane_stats)."""
        return self._read("d3q19_plane_stats", 5 * self.ip.LatticeSize[2], np.float64).reshape(-1, 5)

    def shear_profile(self):
        """(u_mean (Nz, 3), wall shear rate, particle-region shear rate), the
        quantities of the reference's compute_shear_stress, in FP64."""
        um = np.zeros(3 * self.ip.LatticeSize[2], np.float64)
        w, r = C.c_double(), C.c_double()
        self._check(self.lib.d3q19_shear_profile(self.h, _ptr(um), C.byref(w), C.byref(r)), "shear_profile")
        return um.reshape(-1, 3), w.value, r.value

    def mean_stress(self):
        """(mean viscous shear stress, mean shear rate, effective viscosity)."""
        a, b, c = C.c_double(), C.c_double(), C.c_double()
        self._check(self.lib.d3q19_mean_stress(self.h, C.byref(a), C.byref(b), C.byref(c)), "mean_stress")
        return a.value, b.value, c.value

    def checkpoint(self) -> np.ndarray:
        """The whole device state (d3q19_checkpoint) as a uint8 array."""
        n = C.c_size_t()
        self._check(self.lib.d3q19_checkpoint_bytes(self.h, C.byref(n)), "checkpoint_bytes")
        buf = np.zeros(n.value, np.uint8)
        self._check(self.lib.d3q19_checkpoint(self.h, _ptr(buf), buf.nbytes), "checkpoint")
        return buf

    def restore(self, buf):
        """Loads a checkpoint of a context with the same parameters."""
        b = np.ascontiguousarray(buf, np.uint8)
        self._check(self.lib.d3q19_restore(self.h, _ptr(b), b.nbytes), "restore")

    def profile(self, enable: bool):
        self._check(self.lib.d3q19_profile(self.h, int(enable)), "profile")

    def profile_read(self):
        a, b = C.c_double(), C.c_double()
        na, nb = C.c_int(), C.c_int()
        self._check(self.lib.d3q19_profile_read(self.h, C.byref(a), C.byref(na), C.byref(b), C.byref(nb)),
                    "profile_read")
        return a.value, na.value, b.value, nb.value

    @property
    def stream_ptr(self) -> int:
        return int(self.lib.d3q19_stream(self.h) or 0)

    def tau_clamp_count(self) -> int:
        return int(self.lib.d3q19_tau_clamp_count(self.h))

    def close(self):
        if getattr(self, "h", None) and getattr(self, "owned", True):
            self.lib.d3q19_destroy(self.h)
        self.h = None

    @classmethod
    def _view(cls, lib, handle, ip: IntParams, fp: FlpParams, options: Options):
        """A context owned by someone else (a pool member): read-backs only."""
        sim = cls.__new__(cls)
        sim.lib, sim.h, sim.owned = lib, handle, False
        sim.ip = IntParams.from_buffer_copy(bytes(ip))
        sim.fp = FlpParams.from_buffer_copy(bytes(fp))
        sim.options = options
        sim.nc = sim.ip.LatticeSize[0] * sim.ip.LatticeSize[1] * sim.ip.LatticeSize[2]
        sim.np = sim.ip.NumParticles
        sim.nfa = max(sim.ip.WorkGroupsPerParticle, 1)
        sim.nzones = sim.ip.NumZones[0] * sim.ip.NumZones[1] * sim.ip.NumZones[2]
        return sim


def context_bytes(ip: IntParams, options: Options | None = None) -> int:
    """Device memory a context of these parameters allocates (host-side
    arithmetic, no GPU needed)."""
    out = C.c_size_t()
    rc = cuda_lib().d3q19_context_bytes(C.byref(ip), C.byref(options or Options()), C.byref(out))
    if rc:
        raise D3Q19Error(f"d3q19_context_bytes: {STATUS.get(rc, rc)}")
    return int(out.value)


def tune_export() -> str:
    """The settled classes of the grid autotuner's table (d3q19_tune_export)."""
    lib = cuda_lib()
    n = C.c_size_t()
    rc = lib.d3q19_tune_export(None, 0, C.byref(n))
    if rc:
        raise D3Q19Error(f"d3q19_tune_export: {STATUS.get(rc, rc)}")
    buf = C.create_string_buffer(n.value + 1)
    rc = lib.d3q19_tune_export(buf, n.value + 1, C.byref(n))
    if rc:
        raise D3Q19Error(f"d3q19_tune_export: {STATUS.get(rc, rc)}")
    return buf.value.decode()


def tune_import(text: str):
    """Adds settled classes to the autotuner's table (d3q19_tune_import)."""
    rc = cuda_lib().d3q19_tune_import(text.encode())
    if rc:
        raise D3Q19Error(f"d3q19_tune_import: {STATUS.get(rc, rc)}")


def tune_clear():
    cuda_lib().d3q19_tune_clear()


# D3Q19_TUNE_CACHE names a file that keeps the autotuner's table between
# processes: read when the first pool is created, written when a pool closes.
_TUNE_LOADED = False


def _tune_cache_load():
    global _TUNE_LOADED
    path = os.environ.get("D3Q19_TUNE_CACHE")
    if _TUNE_LOADED or not path:
        return
    _TUNE_LOADED = True
    if os.path.exists(path):
        with open(path) as fh:
            tune_import(fh.read())


def _tune_cache_save():
    path = os.environ.get("D3Q19_TUNE_CACHE")
    if path:
        text = tune_export()
        tmp = f"{path}.{os.getpid()}.tmp"
        with open(tmp, "w") as fh:
            fh.write(text)
        os.replace(tmp, path)


class Pool:
    """Many independent shear cells resident on one GPU, advanced together in
    batched persistent kernels (d3q19_pool_* of the C ABI).

    autotune: the persistent grid sizes come from the library's autotuner
    (d3q19_pool_autotune): advances of at least 100 steps time the candidate
    grids of the pool's work class one by one, then keep the fastest."""

    def __init__(self, device: int = 0, storage: int = 0, rebuild_freq: int = 10, max_slots: int = 256,
                 hbm_budget: int = 64 << 30, inplace: bool = False, autotune: bool = True):
        self.lib = cuda_lib()
        _tune_cache_load()
        h = C.c_void_p()
        rc = self.lib.d3q19_pool_create(device, storage, rebuild_freq, max_slots, hbm_budget, C.byref(h))
        if rc:
            raise D3Q19Error(f"d3q19_pool_create: {STATUS.get(rc, rc)}: {self.lib.d3q19_pool_last_error(None).decode()}")
        self.h = h
        self.device = device
        if autotune:
            self._check(self.lib.d3q19_pool_autotune(self.h, 1), "pool_autotune")
        self.storage = storage
        self.inplace = int(inplace)  # members keep one distribution buffer (AA pattern)
        self.max_slots = max_slots
        self.rebuild_freq = rebuild_freq
        self.period = 2 // math.gcd(2, rebuild_freq) * rebuild_freq
        self.members = {}

    def _check(self, rc, what):
        if rc:
            raise D3Q19Error(f"{what}: {STATUS.get(rc, rc)}: {self.lib.d3q19_pool_last_error(self.h).decode()}")

    def admit(self, hs: "HostState", **option_overrides):
        """Admits the solve of a HostState; returns its slot, or None when the
        pool has no room for it now (EBUSY)."""
        opt = Options.from_buffer_copy(bytes(hs.options))
        opt.storage = self.storage
        opt.rebuild_freq = self.rebuild_freq
        opt.inplace = self.inplace
        for k, v in option_overrides.items():
            setattr(opt, k, v)
        slot = C.c_int(-1)
        arrs = [np.ascontiguousarray(x, np.float32) for x in (hs.f, hs.u, hs.tau)]
        if hs.cfg.ip.NumParticles > 0:
            arrs += [np.ascontiguousarray(x, np.float32) for x in (hs.parKin, hs.parForce, hs.parFluidForce,
                                                                  hs.spherePoints)]
            arrs += [np.ascontiguousarray(x, np.int32) for x in (hs.zoneNeighDat, hs.parsZone, hs.zoneMembers,
                                                                hs.numParInZone)]
        else:
            arrs += [None] * 8
        rc = self.lib.d3q19_pool_admit(self.h, C.byref(hs.cfg.ip), C.byref(hs.cfg.fp), C.byref(opt),
                                       *[_ptr(a) for a in arrs], C.byref(slot))
        if rc == EBUSY:
            return None
        self._check(rc, "pool_admit")
        self.members[slot.value] = (IntParams.from_buffer_copy(bytes(hs.cfg.ip)),
                                    FlpParams.from_buffer_copy(bytes(hs.cfg.fp)), opt)
        return slot.value

    def fits(self, hs: "HostState", **option_overrides) -> bool:
        """Whether admit would find a slot and budget for the HostState now
        (host arithmetic only)."""
        opt = Options.from_buffer_copy(bytes(hs.options))
        opt.storage = self.storage
        opt.rebuild_freq = self.rebuild_freq
        opt.inplace = self.inplace
        for k, v in option_overrides.items():
            setattr(opt, k, v)
        used, budget, n = self.usage()
        return n < self.max_slots and used + context_bytes(hs.cfg.ip, opt) <= budget

    def advance(self, nsteps: int):
        self._check(self.lib.d3q19_pool_advance(self.h, nsteps), "pool_advance")

    def member(self, slot: int) -> Simulation:
        """Read-back view of a member (not stepped directly)."""
        hnd = self.lib.d3q19_pool_context(self.h, slot)
        if not hnd:
            raise D3Q19Error(f"pool slot {slot} is free")
        ip, fp, opt = self.members[slot]
        return Simulation._view(self.lib, C.c_void_p(hnd), ip, fp, opt)

    def mean_stress_all(self, max_slots: int):
        """(stress, shear rate, effective viscosity, status) of every slot in one
        pass; status 0 for a healthy member, a negative code for a member
        whose state went non-finite, EINVAL (-1) for a free slot."""
        st, ra, vi = (np.zeros(max_slots, np.float64) for _ in range(3))
        code = np.zeros(max_slots, np.int32)
        self._check(self.lib.d3q19_pool_mean_stress(self.h, _ptr(st), _ptr(ra), _ptr(vi), _ptr(code)),
                    "pool_mean_stress")
        return st, ra, vi, code

    def steps(self, slot: int) -> int:
        return int(self.lib.d3q19_pool_slot_steps(self.h, slot))

    def evict(self, slot: int):
        """Checkpoints the member and frees its slot; returns (checkpoint,
        parameters) for readmit."""
        n = C.c_size_t()
        hnd = self.lib.d3q19_pool_context(self.h, slot)
        if not hnd:
            raise D3Q19Error(f"pool slot {slot} is free")
        self._check(self.lib.d3q19_checkpoint_bytes(C.c_void_p(hnd), C.byref(n)), "checkpoint_bytes")
        buf = np.zeros(n.value, np.uint8)
        self._check(self.lib.d3q19_pool_evict(self.h, slot, _ptr(buf), buf.nbytes), "pool_evict")
        return buf, self.members.pop(slot)

    def readmit(self, evicted):
        """Re-admits an evicted member; returns its slot, or None when the
        pool has no room for it now (EBUSY)."""
        buf, (ip, fp, opt) = evicted
        b = np.ascontiguousarray(buf, np.uint8)
        slot = C.c_int(-1)
        rc = self.lib.d3q19_pool_readmit(self.h, C.byref(ip), C.byref(fp), C.byref(opt), _ptr(b), b.nbytes,
                                         C.byref(slot))
        if rc == EBUSY:
            return None
        self._check(rc, "pool_readmit")
        self.members[slot.value] = (ip, fp, opt)
        return slot.value

    def release(self, slot: int):
        self._check(self.lib.d3q19_pool_release(self.h, slot), "pool_release")
        self.members.pop(slot, None)

    def usage(self):
        used, budget, n = C.c_size_t(), C.c_size_t(), C.c_int()
        self._check(self.lib.d3q19_pool_usage(self.h, C.byref(used), C.byref(budget), C.byref(n)), "pool_usage")
        return int(used.value), int(budget.value), int(n.value)

    def set_grid(self, fluid_blocks: int, particle_blocks: int, contact_blocks: int):
        self._check(self.lib.d3q19_pool_set_grid(self.h, fluid_blocks, particle_blocks, contact_blocks), "set_grid")

    def get_grid(self):
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        self._check(self.lib.d3q19_pool_get_grid(self.h, C.byref(a), C.byref(b), C.byref(c)), "get_grid")
        return a.value, b.value, c.value

    def autotune(self, enable: bool = True):
        self._check(self.lib.d3q19_pool_autotune(self.h, int(enable)), "pool_autotune")

    def tune_state(self) -> dict:
        """The grid in use (CTAs per SM) and the tuner's progress on the
        pool's current work class."""
        v = [C.c_int() for _ in range(5)]
        self._check(self.lib.d3q19_pool_tune_state(self.h, *[C.byref(x) for x in v]), "pool_tune_state")
        return {"fluid_ctas_per_sm": v[0].value, "particle_ctas_per_sm": v[1].value, "settled": bool(v[2].value),
                "tried": v[3].value, "candidates": v[4].value}

    def tune_trials(self) -> list:
        """[(fluid CTAs/SM, particle CTAs/SM, ns per fluid tile step or None)]
        of the pool's current work class."""
        n = C.c_int()
        self._check(self.lib.d3q19_pool_tune_trials(self.h, None, None, None, 0, C.byref(n)), "pool_tune_trials")
        f = np.zeros(n.value, np.int32)
        q = np.zeros(n.value, np.int32)
        t = np.zeros(n.value, np.float64)
        self._check(self.lib.d3q19_pool_tune_trials(self.h, f.ctypes.data, q.ctypes.data, t.ctypes.data, n.value,
                                                    C.byref(n)), "pool_tune_trials")
        return [(int(a), int(b), float(c) if c >= 0 else None) for a, b, c in zip(f, q, t)]

    def synchronize(self):
        self._check(self.lib.d3q19_pool_synchronize(self.h), "pool_synchronize")

    def poll(self) -> bool:
        """Whether the last advance has finished on the device (no wait)."""
        rc = self.lib.d3q19_pool_poll(self.h)
        if rc < 0:
            self._check(rc, "pool_poll")
        return rc == 1

    @property
    def stream_ptr(self) -> int:
        return int(self.lib.d3q19_pool_stream(self.h) or 0)

    def close(self):
        if getattr(self, "h", None):
            self.lib.d3q19_pool_destroy(self.h)
            self.h = None
            _tune_cache_save()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
