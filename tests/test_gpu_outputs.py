"""GPU side of the output and restart files: the mid-plane fields that dasha_midplane gathers
on the device equal the host gather from dasha_get_state and dasha_current bit for bit (the
same FP64 operations on the same values), the m2d file made from them equals the oracle's
text, and a run restored from its restart file continues as the uninterrupted run does."""
import os

import numpy as np
import pytest

from dasha_b200 import capi, harris, restart
from oracle import fortran_io as fio

pytestmark = pytest.mark.gpu

SMALL = harris.RunConfig("small-32x16x32", 32, 16, 32, False, 0.005, 0.5, 4)
RAGGED = harris.RunConfig("ragged-96x12x36-sinh", 96, 12, 36, True, 0.003, 1.0, 4, dt_whistler=1)
# 256x128 planes of 256 KB: the 64 MB transfer chunks hold 256 planes, so 300 planes make two
# chunks per field on the streamed checkpoint and restore
CHUNKS = harris.RunConfig("chunks-256x128x300", 256, 128, 300, False, 0.005, 0.5, 4)


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32"])
@pytest.mark.parametrize("cfg", [SMALL, RAGGED], ids=lambda c: c.name)
def test_midplane_matches_host_gather(cfg, precision):
    d = capi.gem_context(cfg, precision)
    d.run(2)
    mp = d.midplane()
    X, cur = d.get_state(), d.current()
    host = restart.midplane_host(harris.to_halo(X), harris.to_halo(cur))
    assert np.array_equal(mp, host)
    assert np.array_equal(mp, fio.output_fields(X, cur)[:, :, cfg.my // 2, :])
    d.close()


def test_m2d_from_device_plane(tmp_path):
    d = capi.gem_context(SMALL, 0)
    t, _ = d.run(1)
    p = tmp_path / "m2d001.dat"
    restart.write_m2d(str(p), t, d.x, d.z, d.midplane())
    assert p.read_text() == fio.m2d_text(t, d.x, d.z, d.get_state(), d.current())
    d.close()


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32"])
def test_restart_continues_the_run_bit_for_bit(tmp_path, precision):
    """k steps, checkpoint, restore into a fresh context, k more steps == 2k steps, bit for bit
    (survey §5): the restart file holds FP64 totals, from which neither the FP64 perturbation
    split nor the FP32 Kahan pair can be recovered exactly, so the checkpoint also writes the
    exact-resume record <file>.state, which the restore takes when it belongs to the file."""
    a = capi.gem_context(SMALL, precision)
    t, _ = a.run(2)
    path = restart.checkpoint(a, str(tmp_path), ncase=1, nstep=2, time=t, nst=3)
    assert path.endswith("mhd003000") and os.path.exists(path + ".state")
    b = capi.gem_context(SMALL, precision)
    b.run(1)                                                   # another state before the restore
    ncase, nstep, tb, nst = restart.restore(b, str(tmp_path), 3)
    assert (ncase, nstep, tb, nst) == (1, 2, t, 3)
    assert np.array_equal(a.get_state(), b.get_state())
    ta, _ = a.run(2, t, 2)
    tb2, _ = b.run(2, tb, 2)
    assert ta == tb2
    assert np.array_equal(a.get_state(), b.get_state())
    # without the record the file alone restores the state to one rounding (FP64) or to the
    # compensation the file does not carry (FP32)
    os.remove(path + ".state")
    c = capi.gem_context(SMALL, precision)
    restart.restore(c, str(tmp_path), 3)
    a2 = capi.gem_context(SMALL, precision)
    a2.run(2)
    xa, xc = a2.get_state(), c.get_state()
    scale = np.abs(xa).reshape(8, -1).max(axis=1)
    rt = np.abs(xa - xc).reshape(8, -1).max(axis=1) / scale
    assert rt.max() < (1e-15 if precision == 0 else 1e-7), rt
    for x in (a, b, c, a2):
        x.close()


def test_restore_rejects_a_state_record_of_another_checkpoint(tmp_path):
    a = capi.gem_context(SMALL, 1)
    t, _ = a.run(1)
    p1 = restart.checkpoint(a, str(tmp_path), 1, 1, t, 1)
    t2, _ = a.run(1, t, 1)
    p2 = restart.checkpoint(a, str(tmp_path), 1, 2, t2, 2)
    os.replace(p2 + ".state", p1 + ".state")                    # step 2's record beside step 1's file
    b = capi.gem_context(SMALL, 1)
    before = b.get_state()
    with pytest.raises(capi.DashaError) as e:
        restart.restore(b, str(tmp_path), 1)
    assert e.value.code == capi.E_INVALID
    assert np.array_equal(b.get_state(), before)
    a.close()
    b.close()


@pytest.mark.parametrize("maxsub", [0, 1 << 20], ids=["one-subrecord", "1MiB-subrecords"])
@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32"])
@pytest.mark.parametrize("cfg", [SMALL, CHUNKS], ids=lambda c: c.name)
def test_streamed_checkpoint_equals_host_path(tmp_path, cfg, precision, maxsub):
    d = capi.gem_context(cfg, precision)
    t, _ = d.run(1)
    p = restart.checkpoint(d, str(tmp_path), 2, 1, t, 5, max_subrecord=maxsub)
    h = tmp_path / "host"
    restart.checkpoint_host(d, str(h), 2, 1, t, 5, max_subrecord=maxsub)
    assert open(p, "rb").read() == h.read_bytes()
    d.close()


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32"])
@pytest.mark.parametrize("cfg", [SMALL, CHUNKS], ids=lambda c: c.name)
def test_streamed_restore_equals_host_path(tmp_path, cfg, precision):
    a = capi.gem_context(cfg, precision)
    t, _ = a.run(1)
    restart.checkpoint_host(a, str(tmp_path / restart.restart_name(7)), 4, 1, t, 7, max_subrecord=1 << 20)
    b = capi.gem_context(cfg, precision)
    b.run(1)                                                   # a different state before the restore
    assert restart.restore(b, str(tmp_path), 7) == (4, 1, t, 7)
    c = capi.gem_context(cfg, precision)
    assert restart.restore_host(c, str(tmp_path / restart.restart_name(7))) == (4, 1, t, 7)
    assert np.array_equal(b.get_state(), c.get_state())
    for x in (a, b, c):
        x.close()


def test_restore_rejects_a_mismatched_file_and_keeps_the_state(tmp_path):
    a = capi.gem_context(SMALL, 0)
    restart.checkpoint(a, str(tmp_path), 1, 0, 0.0, 1)
    other = harris.RunConfig("small-64x16x32", 64, 16, 32, False, 0.005, 0.5, 4)
    b = capi.gem_context(other, 0)
    before = b.get_state()
    with pytest.raises(capi.DashaError) as e:
        restart.restore(b, str(tmp_path), 1)                   # another grid
    assert e.value.code == capi.E_INVALID
    assert np.array_equal(b.get_state(), before)
    p = tmp_path / restart.restart_name(1)
    p.write_bytes(p.read_bytes()[:-100])                       # truncated
    before = a.get_state()
    with pytest.raises(capi.DashaError) as e:
        restart.restore(a, str(tmp_path), 1)
    assert e.value.code == capi.E_INVALID
    assert np.array_equal(a.get_state(), before)
    a.setdt(0.0)                                               # the context still steps
    a.close()
    b.close()


@pytest.mark.parametrize("cfg", [SMALL, CHUNKS], ids=lambda c: c.name)
def test_stream_out_equals_get_state_and_current(cfg):
    """dasha_stream_out delivers every plane of every field once, fields and planes in order,
    with the values of dasha_get_state / dasha_current (two chunks per field on CHUNKS)."""
    d = capi.gem_context(cfg, 1)
    d.run(1)
    for what, nf, ref in ((0, 8, d.get_state()), (1, 3, d.current())):
        got = np.full((nf, cfg.mz, cfg.my, cfg.mx), np.nan)
        order = []

        def take(m, k0, k1, rows):
            order.append((m, k0, k1))
            got[m, k0:k1] = rows
            return False

        d.stream_out(what, take)
        assert np.array_equal(got, ref)
        assert [o[0] for o in order] == sorted(o[0] for o in order)
        for m in range(nf):
            ks = [(k0, k1) for mm, k0, k1 in order if mm == m]
            assert ks[0][0] == 0 and ks[-1][1] == cfg.mz and all(a[1] == b[0] for a, b in zip(ks, ks[1:]))
    d.close()


def test_stream_out_stops_when_asked():
    d = capi.gem_context(CHUNKS, 0)
    seen = []
    with pytest.raises(capi.DashaError) as e:
        d.stream_out(0, lambda m, k0, k1, rows: seen.append(m) or True)
    assert e.value.code == capi.E_INVALID and seen == [0]
    assert np.isfinite(d.get_state()).all()                     # the context is still usable
    d.close()


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32"])
@pytest.mark.parametrize("cfg", [SMALL, RAGGED], ids=lambda c: c.name)
def test_m3d_from_context_equals_host_path(tmp_path, cfg, precision):
    d = capi.gem_context(cfg, precision)
    t, _ = d.run(1)
    a, b = tmp_path / "m3d_ctx", tmp_path / "m3d_host"
    restart.write_m3d_ctx(d, str(a), t)
    restart.write_m3d(str(b), t, d.x, d.y, d.z, harris.to_halo(d.get_state()), harris.to_halo(d.current()))
    assert a.read_text() == b.read_text()
    d.close()
