"""The reference's on-disk formats (grid, restart file, filestat) as the
library reads and writes them, against oracle/restart_oracle.py, on the CPU.
These functions are host-only: they make no CUDA call.

Byte and record work, so the bar is bit-exact: the library's files equal the
oracle's byte for byte, and values read back equal the FP32 rounding of the
values written.
"""
import numpy as np
import pytest

import restart_oracle as ro


def _lib():
    from desalm import solver
    return solver


def _state(N, seed, turbulence):
    rng = np.random.default_rng(seed)
    q = rng.normal(size=(N, 5))
    qn = rng.normal(size=(N, 5))
    if not turbulence:
        q[:, 4] = 0.0
        qn[:, 4] = 0.0
    nut = rng.uniform(0.0, 1e-3, size=N)
    return q, qn, nut


def _f32(a):
    return np.asarray(a, np.float32).astype(np.float64)


@pytest.mark.parametrize("turbulence", [0, 1])
def test_solu_write_is_the_reference_layout(tmp_path, turbulence):
    S = _lib()
    im, jm, km = 7, 5, 3
    q, qn, nut = _state(im * jm * km, 1 + turbulence, turbulence)
    p = tmp_path / "solu.000"
    S.solu_write(p, im, jm, km, turbulence, q.reshape(-1), qn.reshape(-1), nut)
    assert p.read_bytes() == ro.solu_written(q, qn, nut, turbulence)
    recs = ro.read_records(p.read_bytes())
    assert len(recs) == (11 if turbulence else 8)
    assert all(len(r) == im * jm * km * 4 for r in recs)


@pytest.mark.parametrize("turbulence,layout", [(1, "records"), (0, "records"), (0, "one_record")])
def test_solu_read_both_layouts(tmp_path, turbulence, layout):
    """The reference's reader takes, for a laminar case, q(1..me) as one
    record (src/init.F90:2450-2451) while its writer writes one record per
    component; both are read here."""
    S = _lib()
    im, jm, km = 6, 4, 5
    N = im * jm * km
    q, qn, nut = _state(N, 7, turbulence)
    data = ro.solu_written(q, qn, nut, turbulence) if layout == "records" else ro.solu_as_read(q, qn, nut, turbulence)
    p = tmp_path / "solu"
    p.write_bytes(data)
    got = S.solu_read(p, im, jm, km, turbulence)
    me = ro.me_of(turbulence)
    gq, gqn = got["q"].reshape(N, 5), got["qn"].reshape(N, 5)
    assert np.array_equal(gq[:, :me], _f32(q[:, :me]))
    assert np.array_equal(gqn[:, :me], _f32(qn[:, :me]))
    assert not gq[:, me:].any() and not gqn[:, me:].any()
    if turbulence:
        assert np.array_equal(got["nut"], _f32(nut))


@pytest.mark.parametrize("turbulence", [0, 1])
def test_grid_round_trip_and_bytes(tmp_path, turbulence):
    S = _lib()
    im, jm, km = 5, 4, 6
    N = im * jm * km
    rng = np.random.default_rng(3)
    x, y, z, wd = (rng.normal(size=N) for _ in range(4))
    p = tmp_path / "grid"
    S.grid_write(p, im, jm, km, turbulence, x, y, z, wd if turbulence else None)
    assert p.read_bytes() == ro.grid_bytes(x, y, z, wd, turbulence)
    g = S.grid_read(p, im, jm, km, turbulence)
    for a, b in ((g["x"], x), (g["y"], y), (g["z"], z)):
        assert np.array_equal(a, _f32(b))
    if turbulence:
        assert np.array_equal(g["wd"], _f32(wd))


def test_filestat_round_trip_and_angle_wrap(tmp_path):
    S = _lib()
    p = tmp_path / "filestat"
    S.filestat_write(p, 12.5, 250, [0.25, 7.0])
    text = p.read_text()
    assert ro.filestat_read(text, 2)[:2] == (12.5, 250)
    t, n, ang = S.filestat_read(p, 2)
    assert (t, n) == (12.5, 250)
    want = ro.filestat_read(text, 2)[2]
    assert np.allclose(ang, want, rtol=0, atol=1e-12) and ang[1] < 2 * np.pi


def test_bad_files_are_errors(tmp_path):
    S = _lib()
    im, jm, km = 4, 4, 4
    q, qn, nut = _state(64, 9, 1)
    good = ro.solu_written(q, qn, nut, 1)
    with pytest.raises(S.DesalmError, match="cannot open"):
        S.solu_read(tmp_path / "missing", im, jm, km, 1)
    p = tmp_path / "short"
    p.write_bytes(good[:len(good) // 2])
    with pytest.raises(S.DesalmError):
        S.solu_read(p, im, jm, km, 1)
    p = tmp_path / "wrongsize"
    p.write_bytes(good)
    with pytest.raises(S.DesalmError, match="expected"):
        S.solu_read(p, im, jm, km + 1, 1)
    bad = bytearray(good)
    bad[4 + 64 * 4] ^= 0xFF  # first record's trailing marker
    p = tmp_path / "marker"
    p.write_bytes(bytes(bad))
    with pytest.raises(S.DesalmError, match="marker"):
        S.solu_read(p, im, jm, km, 1)
