"""Restart and output files of libdasha.so (host code, no GPU) against the pure-Python
restatement in oracle/fortran_io.py: the unformatted restart of recrd / readin
(t3dsdsc.f:4814-4861) byte for byte, its gfortran subrecord framing, the readers' rejection of
files that do not match, the ASCII m2d / m3d files of recrd2 / recrd3 (t3dsdsc.f:4965-5412)
character for character, and the eleven output fields of the mid-y plane."""
import ctypes

import numpy as np
import pytest

from dasha_b200 import capi, harris, restart
from oracle import fortran_io as fio


def _state(mx, my, mz, seed=3):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((8, mz, my, mx))
    X[0] = 1.0 + 0.5 * rng.random((mz, my, mx))            # positive density
    cur = rng.standard_normal((3, mz, my, mx)) * 10.0 ** rng.integers(-3, 4, (3, mz, my, mx))
    return X, cur


# --- E editing, hand-derived from the Fortran rules (scale factor 0, optional zero written) ---
KAT_E14_5E3 = [(1.0, "  0.10000E+001"), (-123.456, " -0.12346E+003"), (0.0, "  0.00000E+000"),
               (1e-5, "  0.10000E-004"), (1.23456789e300, "  0.12346E+301"), (-0.0, " -0.00000E+000"),
               (0.999996, "  0.10000E+001"), (9.999996e-100, "  0.10000E-098")]
KAT_E10_4 = [(1.0, "0.1000E+01"), (-1.0, "-.1000E+01"), (0.0, "0.0000E+00"), (1.5e100, "0.1500+101"),
             (-2.5e-120, "-.2500-119"), (0.99996, "0.1000E+01"), (123.456, "0.1235E+03")]


def test_oracle_e_editing_known_answers():
    for v, s in KAT_E14_5E3:
        assert fio.e_edit(v, 14, 5, 3) == s, v
    for v, s in KAT_E10_4:
        assert fio.e_edit(v, 10, 4) == s, v


def test_library_e_editing_known_answers(tmp_path):
    vals = np.array([v for v, _ in KAT_E14_5E3])
    plane = np.zeros((11, 1, vals.size))
    plane[0, 0] = vals
    p = tmp_path / "m2d.dat"
    restart.write_m2d(str(p), 0.0, np.zeros(vals.size), np.zeros(1), plane)
    lines = p.read_text().splitlines()
    i1 = lines.index(f" {1:11d}")
    got = "".join(lines[i1 + 1:i1 + 3])
    assert got == "".join(" " + s for _, s in KAT_E14_5E3)
    # E10.4 through the 3-D writer: the values as x coordinates
    xs = np.array([v for v, _ in KAT_E10_4])
    X = np.ones((8, 1, 1, xs.size))
    H = harris.to_halo(X)
    Hc = harris.to_halo(np.zeros((3, 1, 1, xs.size)))
    p3 = tmp_path / "m3d"
    restart.write_m3d(str(p3), 0.0, xs, np.zeros(1), np.zeros(1), H, Hc)
    line = p3.read_text().splitlines()[2]
    assert line == "".join(" " + s for _, s in KAT_E10_4) + (" " + fio.e_edit(0.0, 10, 4)) * 2   # y, z


def test_oracle_records_round_trip():
    data = bytes(range(256)) * 3
    for maxsub in (fio.GFORTRAN_MAX_SUBRECORD, 100, 7, 1):
        assert fio.read_records(fio.write_record(data, maxsub) + fio.write_record(b"", maxsub)) == [data, b""]
    # gfortran's markers for a record split in three
    b = fio.write_record(b"abcdefgh", 3)
    assert b == (b"\xfd\xff\xff\xffabc\x03\x00\x00\x00" + b"\xfd\xff\xff\xffdef\xfd\xff\xff\xff"
                 + b"\x02\x00\x00\x00gh\xfe\xff\xff\xff")


@pytest.mark.parametrize("maxsub", [0, 4096, 1000, 12])
def test_restart_bytes_match_oracle(tmp_path, maxsub):
    mx, my, mz = 9, 5, 7
    X, _ = _state(mx, my, mz)
    H = restart.restart_array(X)
    p = tmp_path / restart.restart_name(12)
    restart.write_restart(str(p), 3, 4567, 12.375, 12, H, max_subrecord=maxsub)
    ref = fio.restart_bytes(3, 4567, 12.375, 12, H, maxsub or fio.GFORTRAN_MAX_SUBRECORD)
    assert p.read_bytes() == ref
    ncase, nstep, time, nst, H2 = restart.read_restart(str(p), mx, my, mz)
    assert (ncase, nstep, time, nst) == (3, 4567, 12.375, 12)
    assert np.array_equal(H2, H)


def test_restart_padded_leading_dimensions(tmp_path):
    mx, my, mz = 8, 6, 5
    X, _ = _state(mx, my, mz, seed=5)
    H = restart.restart_array(X)
    ld1, ld2 = mx + 9, my + 3
    Hp = np.full((8, mz + 4, ld2, ld1), -7.0)
    Hp[:, :, :my, :mx + 4] = H
    p1, p2 = tmp_path / "a", tmp_path / "b"
    restart.write_restart(str(p1), 1, 2, 3.0, 4, H)
    lib = capi.load()
    assert lib.dasha_restart_write(str(p2).encode(), 1, 2, 3.0, 4, mx, my, mz, capi._dp(Hp), ld1, ld2, 0) == 0
    assert p1.read_bytes() == p2.read_bytes()
    # read back into a padded array: only the (mx+4, my, mz+4) block changes
    out = np.full_like(Hp, 99.0)
    a, b, d, t = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
    assert lib.dasha_restart_read(str(p1).encode(), ctypes.byref(a), ctypes.byref(b), ctypes.byref(t),
                                  ctypes.byref(d), mx, my, mz, capi._dp(out), ld1, ld2) == 0
    assert np.array_equal(out[:, :, :my, :mx + 4], H)
    assert (out[:, :, my:, :] == 99.0).all() and (out[:, :, :, mx + 4:] == 99.0).all()


def test_restart_reader_accepts_any_split_and_rejects_mismatches(tmp_path):
    mx, my, mz = 6, 4, 5
    X, _ = _state(mx, my, mz, seed=9)
    H = restart.restart_array(X)
    p = tmp_path / "f"
    for maxsub in (7, 13, 8 * 1000 + 3):                       # splits inside doubles
        p.write_bytes(fio.restart_bytes(2, 3, 0.5, 1, H, maxsub))
        assert np.array_equal(restart.read_restart(str(p), mx, my, mz)[4], H)
    good = fio.restart_bytes(2, 3, 0.5, 1, H)
    with pytest.raises(capi.DashaError):
        restart.read_restart(str(p), mx + 1, my, mz)          # wrong grid: record 2 too short
    p.write_bytes(good)
    with pytest.raises(capi.DashaError):
        restart.read_restart(str(p), mx, my, mz - 1)          # record 2 too long
    p.write_bytes(good[:-9])
    with pytest.raises(capi.DashaError):
        restart.read_restart(str(p), mx, my, mz)              # truncated
    bad = bytearray(good)
    bad[-1] ^= 1                                              # trailing marker of record 2
    p.write_bytes(bytes(bad))
    with pytest.raises(capi.DashaError):
        restart.read_restart(str(p), mx, my, mz)
    with pytest.raises(capi.DashaError):
        restart.read_restart(str(tmp_path / "missing"), mx, my, mz)


@pytest.mark.parametrize("mx,my,mz,nprx,nprz", [(10, 4, 9, 3, 2), (9, 3, 8, 3, 2), (13, 2, 7, 4, 3), (8, 3, 6, 1, 1)])
def test_rank_files_match_oracle(tmp_path, mx, my, mz, nprx, nprz):
    """A global state split into the rank files of an nprx x nprz run byte for byte as the
    oracle forms them, and the files assembled back into the same interior; the last rank of a
    direction holds the extra node when mx mod nprx (mz mod nprz) is 1."""
    X, _ = _state(mx, my, mz, seed=mx + 10 * mz)
    H = harris.to_halo(X)                                     # NaN halo: it must not be read
    restart.write_restart_ranks(str(tmp_path), 1, 30, 2.5, 4, nprx, nprz, H, max_subrecord=1000)
    for r in range(nprx * nprz):
        ref = fio.restart_bytes(1, 30, 2.5, 4, fio.rank_local(X, r, nprx, nprz), 1000)
        assert (tmp_path / restart.restart_name(4, r)).read_bytes() == ref, r
    ncase, nstep, t, nst, G = restart.read_restart_ranks(str(tmp_path), 4, nprx, nprz, mx, my, mz)
    assert (ncase, nstep, t, nst) == (1, 30, 2.5, 4)
    assert np.array_equal(harris.from_halo(G, mx, my, mz), X)
    # the oracle's gather rule covers every global node exactly once
    hits = np.zeros((mz, mx), int)
    for r in range(nprx * nprz):
        _, gx, _, gz = fio.rank_interior(r, mx, mz, nprx, nprz)
        hits[gz, gx] += 1
    assert (hits == 1).all()


def test_rank_files_read_from_oracle_and_rejected(tmp_path):
    mx, my, mz, nprx, nprz = 10, 3, 9, 3, 2
    X, _ = _state(mx, my, mz, seed=3)
    for r in range(nprx * nprz):                              # files made by the oracle alone
        L = fio.rank_local(X, r, nprx, nprz)
        lx, gx, lz, gz = fio.rank_interior(r, mx, mz, nprx, nprz)
        assert np.array_equal(L[:, lz, :, lx], X[:, gz, :, gx])
        (tmp_path / restart.restart_name(2, r)).write_bytes(fio.restart_bytes(5, 6, 7.0, 2, L, 97))
    G = restart.read_restart_ranks(str(tmp_path), 2, nprx, nprz, mx, my, mz)[4]
    assert np.array_equal(harris.from_halo(G, mx, my, mz), X)
    with pytest.raises(capi.DashaError):
        restart.read_restart_ranks(str(tmp_path), 2, 3, 3, mx, my, mz)     # other process grid: records differ
    with pytest.raises(capi.DashaError):
        restart.read_restart_ranks(str(tmp_path), 2, 4, 2, mx, my, mz)     # mod(10, 4) = 2
    p = tmp_path / restart.restart_name(2, 4)
    p.write_bytes(fio.restart_bytes(5, 6, 7.5, 2, fio.rank_local(X, 4, nprx, nprz)))
    with pytest.raises(capi.DashaError):
        restart.read_restart_ranks(str(tmp_path), 2, nprx, nprz, mx, my, mz)   # another time in one rank


def test_restart_reader_survives_corrupt_files(tmp_path):
    """Random damage to a restart file (bytes flipped in the markers or the data, the file cut
    or extended, markers replaced by extreme lengths): the reader returns the data only when
    the records still hold exactly the grid's bytes, else a status; it never reads past them."""
    mx, my, mz = 6, 3, 5
    X, _ = _state(mx, my, mz, seed=31)
    H = restart.restart_array(X)
    good = fio.restart_bytes(1, 2, 3.0, 4, H, 64)
    rng = np.random.default_rng(99)
    p = tmp_path / "f"
    outcomes = {"ok": 0, "error": 0}
    for trial in range(300):
        b = bytearray(good)
        kind = trial % 4
        if kind == 0:                                     # flip a few bytes anywhere
            for q in rng.integers(0, len(b), rng.integers(1, 4)):
                b[q] ^= int(rng.integers(1, 256))
        elif kind == 1:                                   # cut
            b = b[:int(rng.integers(0, len(b)))]
        elif kind == 2:                                   # extend
            b += bytes(rng.integers(0, 256, int(rng.integers(1, 40))).astype(np.uint8))
        else:                                             # an extreme marker at a marker position
            pos = [0, 4 + 20, 4 + 20 + 4][int(rng.integers(0, 3))]
            b[pos:pos + 4] = int(rng.choice([-2**31, 2**31 - 1, -1, 0, 1 << 30])).to_bytes(4, "little", signed=True)
        p.write_bytes(bytes(b))
        try:
            got = restart.read_restart(str(p), mx, my, mz)
        except capi.DashaError:
            outcomes["error"] += 1
            continue
        outcomes["ok"] += 1
        # accepted only if the records are intact; a flipped data byte changes the values
        recs = fio.read_records(bytes(b), count=2)       # bytes after record 2 are not read
        assert len(recs) >= 2 and len(recs[1]) == H.nbytes
        assert np.ascontiguousarray(got[4]).tobytes() == recs[1]   # bit for bit (a flip may make a NaN)
    assert outcomes["error"] > 100 and outcomes["ok"] > 0


def test_restart_names():
    assert restart.restart_name(7) == "mhd007000"
    assert restart.restart_name(123, 45) == "mhd123045"
    with pytest.raises(ValueError):
        restart.restart_name(1000)


def test_midplane_host_matches_oracle():
    mx, my, mz = 10, 6, 9
    X, cur = _state(mx, my, mz, seed=21)
    got = restart.midplane_host(harris.to_halo(X), harris.to_halo(cur))
    ref = fio.output_fields(X, cur)[:, :, my // 2, :]
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("mx,my,mz", [(10, 6, 9), (7, 3, 11), (1, 1, 1)])
def test_m2d_matches_oracle(tmp_path, mx, my, mz):
    X, cur = _state(mx, my, mz, seed=mx + mz)
    x = np.linspace(-12.8, 12.8, mx)
    z = np.sinh(np.linspace(-3, 3, mz))
    plane = restart.midplane_host(harris.to_halo(X), harris.to_halo(cur))
    p = tmp_path / "m2d001.dat"
    restart.write_m2d(str(p), 17.25, x, z, plane)
    txt = p.read_text()
    assert txt == fio.m2d_text(17.25, x, z, X, cur)
    # list-directed reading back: 0.ddddd, at most half a unit of the 5th digit, 5e-5 relative
    tok = txt.split()
    assert [int(t) for t in tok[:3]] == [2, mx, mz] and float(tok[3]) == 17.25
    vals = np.array([float(t) for t in tok[4:4 + mx + mz]])
    assert np.allclose(vals, np.concatenate([x, z]), rtol=5e-5, atol=0)


def test_m3d_matches_oracle(tmp_path):
    mx, my, mz = 7, 4, 6
    X, cur = _state(mx, my, mz, seed=2)
    x, y, z = np.linspace(0, 1, mx), np.linspace(-2, 2, my), np.linspace(-3, 3, mz)
    p = tmp_path / "m3d004"
    restart.write_m3d(str(p), 3.5, x, y, z, harris.to_halo(X), harris.to_halo(cur))
    assert p.read_text() == fio.m3d_text(3.5, x, y, z, X, cur)


@pytest.mark.parametrize("mx,my,mz", [(1, 1, 12), (11, 1, 3), (3, 1, 5), (2, 2, 9), (13, 7, 2)])
def test_m3d_records_run_across_planes(tmp_path, mx, my, mz):
    """The 3-D writer formats one z plane per piece; records of 11 numbers continue across
    planes of 1, 11, 3, 4 and 91 nodes exactly as in one list."""
    X, cur = _state(mx, my, mz, seed=mx * my + mz)
    x, y, z = np.arange(mx) * 0.5, np.arange(my) - 1.0, np.linspace(-1, 1, mz)
    p = tmp_path / "m3d"
    restart.write_m3d(str(p), 2.0, x, y, z, harris.to_halo(X), harris.to_halo(cur))
    assert p.read_text() == fio.m3d_text(2.0, x, y, z, X, cur)


def test_large_list_parallel_formatting(tmp_path):
    """Lists longer than one formatting block of the library (2^14 lines per thread)."""
    mx, mz = 512, 200
    rng = np.random.default_rng(4)
    plane = rng.standard_normal((11, mz, mx)) * 10.0 ** rng.integers(-120, 120, (11, mz, mx))
    x, z = np.arange(mx, dtype=float), np.arange(mz, dtype=float)
    p = tmp_path / "m2d.dat"
    restart.write_m2d(str(p), 0.0, x, z, plane)
    lines = p.read_text().splitlines()
    i5 = lines.index(f" {5:11d}")
    q = plane[4].reshape(-1)
    body = lines[i5 + 1:i5 + 1 + (q.size + 4) // 5]
    assert len(body) == (q.size + 4) // 5
    for li in rng.integers(0, len(body), 200):
        assert body[li] == fio.format_list(q[5 * li:5 * li + 5], 5, 14, 5, 3).rstrip("\n")


def test_current_dat_lines(tmp_path):
    """diagn's current.dat: a first line, then appended lines, each 7(1X,E13.4)."""
    p = tmp_path / "current.dat"
    rng = np.random.default_rng(8)
    lines = []
    for q in range(3):
        diag = rng.standard_normal(capi.NDIAG) * 10.0 ** rng.integers(-5, 5, capi.NDIAG)
        t = 0.125 * q
        restart.write_current_dat(str(p), diag, t, append=q > 0)
        lines.append(fio.current_dat_line(*diag[3:9], t))
    assert p.read_text() == "".join(lines)
    assert len(lines[0]) == 7 * 14 + 1                        # 7 x (1X + 13 columns) + newline
    restart.write_current_dat(str(p), np.ones(capi.NDIAG), 1.0, append=False)   # starts over
    assert p.read_text() == fio.current_dat_line(*([1.0] * 6), 1.0)
    assert fio.e_edit(-1.0, 13, 4) == "  -0.1000E+01"


def _hard_values(n, seed):
    """Values where a shortcut conversion to 4 or 5 digits would go wrong: random magnitudes
    over 1e-300..1e300, exact decimal ties at the 5th and 6th digit (k + 0.5 and k/10 + 0.05
    scaled by powers of two are not ties; k + 0.5 with 4 and 5 digits are), powers of ten and
    their neighbours, values just below a carry (9.99995e-k), subnormals and extremes."""
    rng = np.random.default_rng(seed)
    v = [rng.uniform(1, 10, n) * 10.0 ** rng.integers(-300, 300, n)]
    v.append(np.concatenate([np.arange(1000, 1100) + 0.5, np.arange(99990, 100000) + 0.5,
                             np.arange(10000, 10100) + 0.5]))
    tens = 10.0 ** np.arange(-300, 301, 7)
    v.append(np.concatenate([tens, np.nextafter(tens, 0), np.nextafter(tens, np.inf)]))
    v.append(9.99995 * 10.0 ** np.arange(-20, 20.0))
    v.append(9.9995 * 10.0 ** np.arange(-20, 20.0))
    v.append(np.array([5e-324, 1e-310, 2.2250738585072014e-308, 1.7976931348623157e308, 1e299, 1e-299]))
    x = np.concatenate(v)
    sgn = np.where(rng.random(x.size) < 0.5, -1.0, 1.0)
    return x * sgn


def test_formatting_matches_exact_decimal_conversion(tmp_path):
    """The library's digits (a double-arithmetic fast path with an exact fallback) against the
    oracle's exact decimal expansion, for E14.5E3 (m2d) and E10.4 (m3d)."""
    vals = _hard_values(3000, 17)
    p = tmp_path / "m2d.dat"
    plane = np.zeros((11, 1, vals.size))
    plane[0, 0] = vals
    restart.write_m2d(str(p), 0.0, np.zeros(vals.size), np.zeros(1), plane)
    lines = p.read_text().splitlines()
    i1 = lines.index(f" {1:11d}")
    got = lines[i1 + 1:i1 + 1 + (vals.size + 4) // 5]
    assert "\n".join(got) + "\n" == fio.format_list(vals, 5, 14, 5, 3)
    p3 = tmp_path / "m3d"
    restart.write_m3d(str(p3), 0.0, vals, np.zeros(1), np.zeros(1), harris.to_halo(np.ones((8, 1, 1, vals.size))),
                      harris.to_halo(np.zeros((3, 1, 1, vals.size))))
    lines = p3.read_text().splitlines()
    got = lines[2:2 + (vals.size + 2 + 10) // 11]
    assert "\n".join(got) + "\n" == fio.format_list(list(vals) + [0.0, 0.0], 11, 10, 4)


def test_step_logs(tmp_path):
    """The main loop's stepnm and unit-20 lines against the oracle, over a run whose step count
    passes 99999 (I5 turns to asterisks there) and whose time passes 99999.99999 (F10.5 does)."""
    KAT_F10_5 = [(0.123456, "   0.12346"), (1234.5, "1234.50000"), (-1234.5, "**********"), (-0.0, "  -0.00000"),
                 (99999.999996, "**********"), (-0.5, "  -0.50000")]
    for v, ref in KAT_F10_5:
        assert fio.f_edit(v, 10, 5) == ref, v
    assert fio.f_edit(0.5, 6, 5) == ".50000" and fio.i_edit(100000, 5) == "*****"
    rng = np.random.default_rng(12)
    sp, dp = tmp_path / "stepnm", tmp_path / "fort.20"
    want_s, want_d = [], []
    steps = list(rng.integers(0, 99998, 40)) + [99998, 99999, 100000, 123456]
    for nstep in steps:
        dt = float(10.0 ** rng.uniform(-6, 0))
        time = float(rng.uniform(0, 2e5)) if nstep > 50000 else float(rng.uniform(0, 100))
        restart.write_step_logs(str(sp), str(dp), int(nstep), time, dt)
        want_s.append(fio.stepnm_line(int(nstep), time, dt))
        want_d.append(fio.dtlog_line(dt, time + dt, int(nstep) + 1))
    assert sp.read_text() == "".join(want_s)
    assert dp.read_text() == "".join(want_d)
    assert "*****" in dp.read_text() and "**********" in dp.read_text()


def test_bad_arguments_rejected(tmp_path):
    lib = capi.load()
    assert lib.dasha_restart_write(None, 0, 0, 0.0, 0, 4, 4, 4, None, 8, 4, 0) == capi.E_INVALID
    H = np.zeros((8, 8, 4, 8))
    assert lib.dasha_restart_write(str(tmp_path / "a").encode(), 0, 0, 0.0, 0, 4, 4, 4, capi._dp(H), 7, 4, 0) == capi.E_INVALID
    assert lib.dasha_restart_write(str(tmp_path / "a").encode(), 0, 0, 0.0, 0, 4, 4, 4, capi._dp(H), 8, 4, -1) == capi.E_INVALID
    assert lib.dasha_m2d_write(str(tmp_path / "m").encode(), 0, 4, 0.0, None, None, None) == capi.E_INVALID
    assert lib.dasha_midplane(None, None) == capi.E_INVALID
    assert lib.dasha_checkpoint(None, b"x", 0, 0, 0.0, 0, 0) == capi.E_INVALID
    assert lib.dasha_stream_out(None, 0, None, None) == capi.E_INVALID
    assert lib.dasha_m3d_write_ctx(None, b"x", 0.0) == capi.E_INVALID
    i, t = ctypes.c_int(), ctypes.c_double()
    assert lib.dasha_restore(None, b"x", ctypes.byref(i), ctypes.byref(i), ctypes.byref(t), ctypes.byref(i)) == capi.E_INVALID
    assert lib.dasha_restart_write(str(tmp_path / "no" / "dir").encode(), 0, 0, 0.0, 0, 4, 4, 4, capi._dp(H), 8, 4, 0) == capi.E_INVALID


class _HostGroup:
    """A stand-in for a z-slab group (dasha_b200/slabs.py SlabGroup): the whole-grid state and
    current as host arrays, and the marker that sends the output helpers down the host path."""
    host_outputs = True

    def __init__(self, mx, my, mz):
        self.x, self.y, self.z = harris.make_grid(mx, my, mz, True)
        self.mx, self.my, self.mz = mx, my, mz
        self.X, self.cur = _state(mx, my, mz, seed=11)

    def get_state(self):
        return self.X.copy()

    def set_state(self, X):
        self.X = np.array(X)

    def current(self):
        return self.cur.copy()


def test_group_outputs_through_host_copies(tmp_path):
    """restart.checkpoint / restore / write_m3d_ctx on a slab group write and read the files the
    host helpers write for the same arrays."""
    g = _HostGroup(12, 4, 9)
    path = restart.checkpoint(g, str(tmp_path), 2, 30, 1.25, 4)
    ref = tmp_path / "ref"
    restart.write_restart(str(ref), 2, 30, 1.25, 4, restart.restart_array(g.X))
    assert path.endswith("mhd004000") and open(path, "rb").read() == ref.read_bytes()
    X0 = g.X.copy()
    g.X = np.zeros_like(g.X)
    assert restart.restore(g, str(tmp_path), 4) == (2, 30, 1.25, 4)
    # the file holds v = (rho v)/rho; the state comes back as rho v to within rounding
    np.testing.assert_allclose(g.X, X0, rtol=1e-14, atol=1e-14)
    restart.write_m3d_ctx(g, str(tmp_path / "m3d_group"), 1.25)
    restart.write_m3d(str(tmp_path / "m3d_host"), 1.25, g.x, g.y, g.z, harris.to_halo(g.X), harris.to_halo(g.cur))
    assert (tmp_path / "m3d_group").read_bytes() == (tmp_path / "m3d_host").read_bytes()
