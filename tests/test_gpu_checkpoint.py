"""Checkpoints (d3q19_checkpoint / d3q19_restore) and pool pre-emption
(d3q19_pool_evict / d3q19_pool_readmit) on the GPU.

* A context restored from a checkpoint continues bit for bit like the one
  it came from: FP32, FP16 storage, the FP64 build and FP64 particles.
* A checkpoint is refused for a context left between passes and by a
  context of other parameters; a truncated or foreign buffer is refused.
* A pool member that is evicted, waits while the others run, and is
  re-admitted ends bit for bit where a member that was never evicted ends;
  the members that stayed are unaffected.
"""
import numpy as np
import pytest

import d3q19_b200 as d3
from d3q19_b200 import serving as sv

pytestmark = pytest.mark.gpu

SUSP = sv.ShearRequest(rid=0, edge=(34, 34, 34), phi=0.2, model="power_law", wall_speed=0.03, seed=7)
OTHER = sv.ShearRequest(rid=1, edge=(36, 36, 36), phi=0.15, model="casson", wall_speed=0.02, seed=8)


def sim_state(sim):
    out = {"u": sim.read_u(), "tau": sim.read_tau(), "f": sim.read_f()}
    if sim.np > 0:
        out["kin"] = sim.read_parkin()
        out["pf"] = sim.read_parforce()
        out["pff"] = sim.read_parfluidforce()
        out["zones"] = np.concatenate(sim.read_zones())
        out["cells"] = sim.read_marker_cells()
    return out


def bits_equal(a, b):
    for k in a:
        x, y = np.ascontiguousarray(a[k]), np.ascontiguousarray(b[k])
        assert x.shape == y.shape and np.array_equal(x.view(np.uint8), y.view(np.uint8)), k


@pytest.mark.parametrize("over", [dict(), dict(storage=1), dict(arithmetic=2), dict(particle_precision=1)],
                         ids=["fp32", "fp16", "fp64-build", "fp64-particles"])
def test_restore_continues_bit_for_bit(over):
    hs = sv.host_state(SUSP)
    a = d3.Simulation.from_host_state(hs, **over)
    a.run(1, 30)  # a zone rebuild at 30; the checkpoint carries the lists
    ck = a.checkpoint()
    a.run(31, 25)
    want = sim_state(a)
    if "particle_precision" in over or "arithmetic" in over:
        want["kin64"] = a.read_parkin64()
    clamps = a.tau_clamp_count()
    a.close()

    b = d3.Simulation.from_host_state(sv.host_state(SUSP), **over)
    b.run(1, 4)  # a different state (and buffer parity) that the restore overwrites
    b.restore(ck)
    b.run(31, 25)
    got = sim_state(b)
    if "kin64" in want:
        got["kin64"] = b.read_parkin64()
    assert b.tau_clamp_count() == clamps
    b.close()
    bits_equal(want, got)


def test_restore_with_step_by_step_calls():
    # A checkpoint taken after d3q19_step calls restores into a context that
    # continues through the graph path (d3q19_run), and the other way round.
    hs = sv.host_state(SUSP)
    a = d3.Simulation.from_host_state(hs)
    for t in range(1, 13):
        a.step(t)
    ck = a.checkpoint()
    a.run(13, 18)
    want = sim_state(a)
    a.close()
    b = d3.Simulation.from_host_state(hs)
    b.restore(ck)
    for t in range(13, 31):
        b.step(t)
    bits_equal(want, sim_state(b))
    b.close()


def test_checkpoint_refusals():
    hs = sv.host_state(SUSP)
    a = d3.Simulation.from_host_state(hs)
    a.run(1, 10)
    ck = a.checkpoint()
    # Between passes of step 11.
    a.lib.d3q19_k_collide_stream(a.h, 11)
    with pytest.raises(d3.D3Q19Error, match="ESTATE"):
        a.checkpoint()
    a.lib.d3q19_k_particles(a.h, 11)
    a.lib.d3q19_k_contacts(a.h, 11)
    a.checkpoint()  # whole again
    # Truncated and foreign buffers.
    with pytest.raises(d3.D3Q19Error, match="EINVAL"):
        a.restore(ck[: len(ck) - 16])
    bad = ck.copy()
    bad[:8] = 0
    with pytest.raises(d3.D3Q19Error, match="EINVAL"):
        a.restore(bad)
    a.close()
    # A context of other parameters.
    c = d3.Simulation.from_host_state(sv.host_state(OTHER))
    with pytest.raises(d3.D3Q19Error, match="EINVAL"):
        c.restore(ck)
    c.close()
    # A context of other options (FP16 storage).
    d = d3.Simulation.from_host_state(hs, storage=1)
    with pytest.raises(d3.D3Q19Error, match="EINVAL"):
        d.restore(ck)
    d.close()


def pool_state(pool, slot):
    m = pool.member(slot)
    return {"u": m.read_u(), "tau": m.read_tau(), "kin": m.read_parkin(), "pff": m.read_parfluidforce(),
            "stress": np.array(m.mean_stress())}


@pytest.mark.parametrize("storage", [0, 1])
def test_pool_evict_and_readmit(storage):
    pool = d3.Pool(storage=storage, max_slots=4)
    sa = pool.admit(sv.host_state(SUSP))
    sb = pool.admit(sv.host_state(OTHER))
    pool.advance(40)
    used_before = pool.usage()[0]
    ev = pool.evict(sa)
    assert pool.usage()[0] < used_before and pool.usage()[2] == 1
    pool.advance(60)  # the other member runs on alone
    sa2 = pool.readmit(ev)
    assert pool.steps(sa2) == pool.period + 40
    pool.advance(40)
    assert pool.steps(sa2) == pool.period + 80 and pool.steps(sb) == pool.period + 140
    got_a, got_b = pool_state(pool, sa2), pool_state(pool, sb)
    pool.close()

    ref = d3.Pool(storage=storage, max_slots=4)
    ra = ref.admit(sv.host_state(SUSP))
    ref.advance(80)
    want_a = pool_state(ref, ra)
    ref.close()
    ref = d3.Pool(storage=storage, max_slots=4)
    rb = ref.admit(sv.host_state(OTHER))
    ref.advance(140)
    want_b = pool_state(ref, rb)
    ref.close()
    bits_equal(want_a, got_a)
    bits_equal(want_b, got_b)


def test_pool_readmit_refusals():
    pool = d3.Pool(storage=0, max_slots=1)
    s = pool.admit(sv.host_state(SUSP))
    pool.advance(20)
    ev = pool.evict(s)
    s2 = pool.admit(sv.host_state(OTHER))
    assert pool.readmit(ev) is None  # the only slot is taken: EBUSY
    pool.release(s2)
    # A checkpoint out of the pool's phase is refused.
    a = d3.Simulation.from_host_state(sv.host_state(SUSP), rebuild_freq=10)
    a.run(1, 7)
    odd = (a.checkpoint(), ev[1])
    a.close()
    with pytest.raises(d3.D3Q19Error, match="EINVAL"):
        pool.readmit(odd)
    assert pool.readmit(ev) is not None
    pool.close()


def _ckpt_layout(ck):
    """Byte offsets of the integer tables of an FP32 checkpoint with spheres
    (header: magic, version, storage, p64, arithmetic, NC, ntiles, np, nfa, P,
    cap, nzones, f_state, last_t, sticky, inplace, phase, clamps)."""
    import struct

    (_, _, storage, p64, arith, NC, ntiles, npar, nfa, P, cap, Z, _, _, _, _, _, _) = struct.unpack_from(
        "<8s4i2q5i3i2iq", ck.tobytes(), 0)
    assert storage == 0 and p64 == 0 and arith == 0
    M = npar * P
    sizes = [("f", 4 * 19 * NC), ("u", 12 * NC), ("tau", 4 * NC), ("kin", 64 * npar), ("pf", 32 * npar),
             ("pff", 32 * npar * nfa), ("sphere", 16 * P), ("mrec", 32 * M), ("tile_count", 4 * ntiles),
             ("tile_list", 4 * ntiles * cap), ("fmax", 8), ("znd", 4 * 28 * Z), ("parsZone", 4 * npar),
             ("zoneMembers", 4 * Z * npar), ("numParInZone", 4 * Z), ("revStart", 4 * (Z + 1)),
             ("revList", 4 * 27 * Z), ("zoneOf", 4 * npar)]
    off, out = 88, {}
    for name, n in sizes:
        out[name] = off
        off += n
    assert off == len(ck)
    return out, dict(np=npar, Z=Z, cap=cap, ntiles=ntiles)


@pytest.mark.parametrize("damage", ["zone_member", "tile_list", "reverse_table", "neighbour_count", "neighbour_id",
                                    "pars_zone", "zone_of"])
def test_restore_refuses_damaged_tables(damage):
    # A checkpoint's integer tables index device arrays: a damaged entry is
    # refused on the host before anything is uploaded.
    hs = sv.host_state(SUSP)
    a = d3.Simulation.from_host_state(hs)
    a.run(1, 10)
    ck = a.checkpoint()
    off, dims = _ckpt_layout(ck)
    ints = lambda name, n: np.frombuffer(ck, np.int32, count=n, offset=off[name])
    bad = ck.copy()
    view = lambda name, n: bad[off[name]:off[name] + 4 * n].view(np.int32)  # noqa: E731  (writable)
    if damage == "zone_member":
        nin = ints("numParInZone", dims["Z"])
        z = int(np.argmax(nin > 0))
        view("zoneMembers", dims["Z"] * dims["np"])[z * dims["np"]] = dims["np"] + 7
    elif damage == "tile_list":
        cnt = ints("tile_count", dims["ntiles"])
        T = int(np.argmax(cnt > 0))
        assert cnt[T] > 0
        view("tile_list", dims["ntiles"] * dims["cap"])[T * dims["cap"]] = -3
    elif damage == "reverse_table":
        view("revStart", dims["Z"] + 1)[dims["Z"]] = 27 * dims["Z"] + 5
    elif damage == "neighbour_count":
        view("znd", 28 * dims["Z"])[0] = 99
    elif damage == "neighbour_id":
        znd = ints("znd", 28 * dims["Z"])
        assert znd[0] > 0
        view("znd", 28 * dims["Z"])[1] = dims["Z"] + 2
    elif damage == "pars_zone":
        view("parsZone", dims["np"])[0] = dims["Z"] + 3
    else:
        view("zoneOf", dims["np"])[0] = -1
    with pytest.raises(d3.D3Q19Error, match="damaged"):
        a.restore(bad)
    a.restore(ck)  # the intact one still restores
    a.run(11, 5)
    a.synchronize()
    a.close()


@pytest.mark.parametrize("field,value", [("phase", 5), ("f_state", 7), ("last_t", -4)])
def test_restore_refuses_damaged_header(field, value):
    # The header's layout phase, distribution state and step are checked
    # before anything is uploaded (an in-place context: the phase selects
    # its buffer).
    import struct

    hs = sv.host_state(SUSP)
    a = d3.Simulation.from_host_state(hs, inplace=1)
    a.run(1, 11)
    ck = a.checkpoint()
    off = {"f_state": 60, "last_t": 64, "phase": 76}[field]
    bad = ck.copy()
    bad[off:off + 4] = np.frombuffer(struct.pack("<i", value), np.uint8)
    with pytest.raises(d3.D3Q19Error):
        a.restore(bad)
    a.restore(ck)
    a.run(12, 5)
    a.synchronize()
    a.close()
