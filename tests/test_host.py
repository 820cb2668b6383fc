"""Host side (C host library and the C ABI's host-only entry points), no GPU:
input parsing with the reference's keyword semantics, the initial state the
reference's host builds, zone tables, periodic map, unit-sphere partitions
and the output writers, all against the reference's own golden data."""
import ctypes as C
import os
import re
import tempfile

import numpy as np
import pytest

from conftest import GOLDEN, REPO, load_golden
from cases import CASES, input_keywords

import d3q19_b200 as d3


def partitions_dir():
    """A directory holding the reference's unit-sphere partition files,
    written from the fixture (tests/golden/make_partitions.py)."""
    d = tempfile.mkdtemp(prefix="usp_")
    os.makedirs(os.path.join(d, "unit_sphere_partitions"))
    with np.load(os.path.join(GOLDEN, "unit_sphere_partitions.npz")) as z:
        for k in z.files:
            with open(os.path.join(d, "unit_sphere_partitions", f"unit_sphere_partition_{k[1:]}.txt"), "wb") as fh:
                fh.write(z[k].tobytes())
    return d


@pytest.fixture(scope="module")
def usp_dir():
    return partitions_dir()


def host_state(name, data_dir, **over):
    cfg = d3.parse_config(d3.keywords_text(dict(input_keywords(CASES[name]), **over)))
    return d3.HostState(cfg, data_dir=data_dir)


@pytest.mark.parametrize("name", sorted(CASES))
def test_initial_state_matches_reference(name, usp_dir):
    """Parsing + initialize_lattice_fields + initialize_particle_fields +
    initialize_particle_zones reproduce the reference host's buffers."""
    g = load_golden(name)
    hs = host_state(name, usp_dir, iterations=0)  # the golden initial state is the iterations=0 run
    ref_ip = d3.IntParams.from_buffer_copy(bytes(g["intDat"]))
    ref_fp = d3.FlpParams.from_buffer_copy(bytes(g["flpDat"]))
    ip, fp = hs.cfg.ip, hs.cfg.fp
    # Every field the kernels read (the reference leaves InterpOrderIBM,
    # MaintainShear and ParForceParams[1] uninitialised).
    for f in ("MaxIterations", "LatticeSize", "SystemSize", "BufferSize", "BoundaryConds", "NumZones",
              "ViscosityModel", "NumParticles", "ParForceModel", "MaxSurfPointsPerNode", "PointsPerParticle",
              "PointsPerWorkGroup", "TotalSurfPoints", "WorkGroupsPerParticle", "BasisVel"):
        assert np.array_equal(np.ctypeslib.as_array(getattr(ip, f)) if not isinstance(getattr(ip, f), int)
                              else getattr(ip, f), np.ctypeslib.as_array(getattr(ref_ip, f))
                              if not isinstance(getattr(ref_ip, f), int) else getattr(ref_ip, f)), f
    for f in ("ConstBodyForce", "EqWeights", "VelUpper", "VelLower", "NewtonianTau", "ViscosityParams",
              "ZoneWidth", "ParticleDiam", "ParticleMass", "PointArea", "ParticleMomInertia", "ParticleZBuffer",
              "DirectForcingCoeff"):
        a, b = getattr(fp, f), getattr(ref_fp, f)
        a = np.array(a if isinstance(a, float) else list(a), np.float32)
        b = np.array(b if isinstance(b, float) else list(b), np.float32)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), f
    assert fp.ParForceParams[0] == ref_fp.ParForceParams[0]
    assert np.array_equal(hs.f.view(np.uint32), g["init_f"].view(np.uint32))
    assert np.array_equal(hs.u, g["init_u"])
    assert np.array_equal(hs.tau, g["init_tau_lb"])
    np_ = ip.NumParticles
    if np_:
        assert np.array_equal(hs.parKin.view(np.uint32), g["init_parKin"].view(np.uint32))
        assert np.array_equal(hs.spherePoints.view(np.uint32), g["init_spherePoints"].view(np.uint32))
        assert np.array_equal(hs.parsZone, g["init_parsZone"])
        assert np.array_equal(hs.numParInZone, g["init_numParInZone"])
        valid = g["init_zoneMembers"] >= 0
        assert np.array_equal(hs.zoneMembers[valid], g["init_zoneMembers"][valid])
        assert np.array_equal(hs.numParInThread, g["init_numParInThread"])
        tv = g["init_threadMembers"] >= 0
        assert np.array_equal(hs.threadMembers[tv], g["init_threadMembers"][tv])
        Z = ip.NumZones[0] * ip.NumZones[1] * ip.NumZones[2]
        for z in range(Z):
            c = g["init_zoneNeighDat"][28 * z]
            assert np.array_equal(hs.zoneNeighDat[28 * z: 28 * z + 1 + c], g["init_zoneNeighDat"][28 * z: 28 * z + 1 + c])


@pytest.mark.parametrize("name", sorted(CASES))
def test_periodic_map_from_library_without_gpu(name):
    g = load_golden(name)
    ip = d3.IntParams.from_buffer_copy(bytes(g["intDat"]))
    assert np.array_equal(d3.periodic_map(ip), g["init_strMap"])


def test_parser_keyword_semantics():
    # Defaults are the reference's table (D3Q19-OpenCL.c:31-64).
    cfg = d3.parse_config("")
    assert cfg.ip.MaxIterations == 1000 and list(cfg.ip.LatticeSize) == [32, 32, 32]
    assert cfg.fp.NewtonianTau == 1.0 and cfg.ip.MaxSurfPointsPerNode == 8
    assert cfg.hp.InitialDist == b"zero" and list(cfg.hp.DomainDecomp) == [2, 2, 2]
    assert cfg.fp.ParForceParams[0] == 1.0 and cfg.fp.ParticleZBuffer == 10.0
    # A line sets every keyword it contains as a substring.
    cfg = d3.parse_config("ovito_xyz_video_freq 1234\n")
    assert cfg.hp.VideoFreq == 1234
    # maintain_shear_rate is a three-int keyword stored at MaintainShear: it
    # also writes ViscosityModel and NumParticles (D3Q19-OpenCL.c:45, 636-641).
    cfg = d3.parse_config("viscosity_model 2\nnum_particles 5\nmaintain_shear_rate 1 3 7\n")
    assert (cfg.ip.MaintainShear, cfg.ip.ViscosityModel, cfg.ip.NumParticles) == (1, 3, 7)
    cfg = d3.parse_config("maintain_shear_rate 1 3 7\nviscosity_model 2\nnum_particles 5\n")
    assert (cfg.ip.ViscosityModel, cfg.ip.NumParticles) == (2, 5)
    # particle_collision_params reads one float (D3Q19-OpenCL.c:56).
    cfg = d3.parse_config("particle_collision_params 2.5 7.0\n")
    assert cfg.fp.ParForceParams[0] == 2.5
    # The reference's own input files parse.
    cfg = d3.parse_config("iterations 100\ntotal_lattice_size 96 96 96\ninitial_f constant\ncpu_only_mode 0\n")
    assert cfg.ip.MaxIterations == 100 and cfg.hp.InitialDist == b"constant"
    # New keywords.
    cfg = d3.parse_config("use_constant_viscosity 0\nibm_points_per_particle 512\nfixed_particles 1\n"
                          "particle_seed 7\nmin_particle_gap 2.0\ntau_max 2.0\ntau_min 0.55\n")
    assert cfg.hp.UseConstantViscosity == 0 and cfg.hp.PointsOverride == 512 and cfg.hp.FixedParticles == 1
    assert cfg.hp.ParticleSeed == 7 and cfg.hp.MinParticleGap == 2.0
    assert cfg.hp.TauMax == 2.0 and abs(cfg.hp.TauMin - 0.55) < 1e-7
    # No new keyword is a substring of a reference line or contains one.
    host_src = open(os.path.join(REPO, "dispersion-shear_d3q19-opencl_b200", "host", "d3q19_host.c")).read()
    keys = re.findall(r'\{"([a-z_0-9]+)", T_', host_src)
    for a in keys:
        for b in keys:
            if a != b:
                assert a not in b, (a, b)


def test_generated_partitions_match_the_reference_files():
    """The recursive zonal equal-area points printed to 5 significant
    digits are the shipped files, except that the files for 256, 512 and
    1024 points store the south pole's x as 0 instead of 1.2246e-16."""
    with np.load(os.path.join(GOLDEN, "unit_sphere_partitions.npz")) as z:
        for k in z.files:
            n = int(k[1:])
            lines = [ln for ln in z[k].tobytes().decode().split("\n") if ln.strip()]
            pts = d3.eqsp_points(n)
            mine = [",".join("%.5g" % c for c in p) for p in pts]
            diff = [i for i, (a, b) in enumerate(zip(lines, mine)) if a.strip() != b]
            if n in (256, 512, 1024):
                assert diff == [n - 1] and lines[-1].strip() == "0,0,-1"
            else:
                assert diff == []


def test_sphere_discretisation_without_files_uses_generated_points(usp_dir):
    cfg = d3.parse_config("num_particles 1\nparticle_diameter 6.0\n")
    a = d3.HostState(cfg, data_dir=usp_dir)
    cfg2 = d3.parse_config("num_particles 1\nparticle_diameter 6.0\n")
    b = d3.HostState(cfg2, data_dir=tempfile.mkdtemp())
    assert a.cfg.ip.PointsPerParticle == b.cfg.ip.PointsPerParticle == 128
    assert np.array_equal(a.spherePoints, b.spherePoints)


def test_rsa_placement_is_seeded_and_respects_gap():
    txt = ("total_lattice_size 64 64 64\nboundary_conditions_xyz 0 0 1\nnum_particles 30\nparticle_diameter 8.0\n"
           "initial_particle_distribution 4\nparticle_seed 3\nmin_particle_gap 2.0\ninitial_particle_buffer 0.0\n"
           "z_wall_particle_buffer 5.0\ndomain_decomposition 1 1 1\n")
    a = d3.HostState(d3.parse_config(txt), data_dir=tempfile.mkdtemp())
    b = d3.HostState(d3.parse_config(txt), data_dir=tempfile.mkdtemp())
    assert np.array_equal(a.parKin, b.parKin)
    c = d3.HostState(d3.parse_config(txt.replace("particle_seed 3", "particle_seed 4")), data_dir=tempfile.mkdtemp())
    assert not np.array_equal(a.parKin, c.parKin)
    x = a.parKin.reshape(-1, 4)[:30, :3].astype(np.float64)
    S = np.array(list(a.cfg.ip.SystemSize), np.float64)
    d = np.abs(x[:, None] - x[None])
    for ax in (0, 1):
        d[..., ax] = np.minimum(d[..., ax], S[ax] - d[..., ax])
    r = np.sqrt((d ** 2).sum(-1)) + np.eye(30) * 1e9
    assert r.min() >= 10.0 - 1e-4
    assert x[:, 2].min() >= 5.0 and x[:, 2].max() <= S[2] - 5.0


@pytest.mark.parametrize("name", ["couette", "sphere_wrap"])
def test_output_writers_match_reference_files(name, usp_dir):
    g = load_golden(name)
    hs = host_state(name, usp_dir)
    h = d3.host_lib()
    d = tempfile.mkdtemp()
    fld, ctr, prof = (os.path.join(d, x) for x in ("field.txt", "centerline.txt", "profile.txt"))
    assert h.d3q19h_write_lattice_field(C.byref(hs.cfg), g["final_u"].ctypes.data_as(C.c_void_p), fld.encode(),
                                        ctr.encode()) == 0
    for fn, key in ((fld, "file_velocity_field_final.txt"),
                    (ctr, "file_matlab_postproc__velocity_field_centerline.txt")):
        assert open(fn, "rb").read() == g[key].tobytes()
    if "file_velocity_profile_z.txt" in g:
        st = (C.c_int * 3)()
        h.d3q19h_compute_shear_stress(C.byref(st), C.byref(hs.cfg), g["final_u"].ctypes.data_as(C.c_void_p),
                                      prof.encode())
        assert open(prof, "rb").read() == g["file_velocity_profile_z.txt"].tobytes()
    if "file_xyz_ovito_output.txt" in g:
        # The last frame of the video file is written from the final state.
        ref = g["file_xyz_ovito_output.txt"].tobytes().decode()
        n_last = int(g["iterations"])
        last = ref[ref.rindex(ref.split("\n")[0] + "\nD3Q19_output, frame %d" % n_last):]
        libc = C.CDLL(None)
        libc.fopen.restype = C.c_void_p
        libc.fopen.argtypes = [C.c_char_p, C.c_char_p]
        libc.fclose.argtypes = [C.c_void_p]
        vid = os.path.join(d, "vid.txt")
        fh = libc.fopen(vid.encode(), b"w")
        h.d3q19h_continuous_output.argtypes = [C.POINTER(d3.Config), C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
        kin = g["final_parKin"] if hs.cfg.ip.NumParticles else np.zeros(4, np.float32)
        h.d3q19h_continuous_output(C.byref(hs.cfg), g["final_u"].ctypes.data_as(C.c_void_p),
                                   kin.ctypes.data_as(C.c_void_p), fh, n_last)
        libc.fclose(fh)
        assert open(vid).read() == last


def _sphere_config(d=8.0):
    kw = dict(total_lattice_size=(24, 24, 24), boundary_conditions_xyz=(0, 0, 1), num_particles=1,
              particle_diameter=d, initial_particle_distribution=3, initial_particle_buffer=11.0,
              domain_decomposition=(1, 1, 1))
    return d3.parse_config(d3.keywords_text(kw))


@pytest.mark.parametrize("defect", ["truncated", "off_sphere", "not_numbers"])
def test_malformed_partition_file_is_rejected(defect):
    # The reference prints and exits on a malformed sphere file
    # (D3Q19-OpenCL.c:598-601); here the host set-up returns an error the
    # caller sees, before any device work.
    cfg = _sphere_config()
    P = 256  # 2^ceil(log2(pi d^2)) for d = 8
    d = tempfile.mkdtemp(prefix="d3q19usp_")
    os.makedirs(os.path.join(d, "unit_sphere_partitions"))
    pts = np.zeros((P, 3))
    pts[:, 2] = 1.0
    lines = [f"{x:.5g},{y:.5g},{z:.5g}" for x, y, z in pts]
    if defect == "truncated":
        lines = lines[:100]
    elif defect == "off_sphere":
        lines[37] = "1.2,0,0"
    else:
        lines[5] = "a,b,c"
    with open(os.path.join(d, "unit_sphere_partitions", f"unit_sphere_partition_{P}.txt"), "w") as fh:
        fh.write("\n".join(lines) + "\n")
    with pytest.raises(d3.D3Q19Error, match="malformed"):
        d3.HostState(cfg, data_dir=d)


def test_well_formed_partition_file_is_used():
    cfg = _sphere_config()
    P = 256
    d = tempfile.mkdtemp(prefix="d3q19usp_")
    os.makedirs(os.path.join(d, "unit_sphere_partitions"))
    with open(os.path.join(d, "unit_sphere_partitions", f"unit_sphere_partition_{P}.txt"), "w") as fh:
        fh.write("0,0,1\n" * P)
    hs = d3.HostState(cfg, data_dir=d)
    sp = hs.spherePoints.reshape(P, 4)
    assert np.allclose(sp[:, :3], [0.0, 0.0, 4.0])  # unit points scaled by d/2
