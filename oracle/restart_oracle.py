"""numpy restatement of the reference's on-disk formats (grid, restart file,
filestat) for one block.

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the library's
readers and writers (des-alm_b200/csrc/restart.cpp).  The product never loads
it.

The reference writes and reads Fortran unformatted sequential files: each
record is a 4-byte little-endian byte count, the payload, and the count again
(the compiler's record format; gfortran and the Intel compiler both use 4-byte
markers by default).  Its reals are real(rdf) = FP32 (src/precision.F90:11),
arrays are stored i fastest.  The reference ships no such files, so parity is
unpinned: these functions restate the loops of the cited routines.

Host arrays follow the library's ABI: q as an (N, 5) array (component
fastest in memory), grids and nu_t as (N,) arrays, N = im * jm * km.
"""
import numpy as np


def record(payload):
    """One Fortran sequential record around the given bytes."""
    n = np.array([len(payload)], "<i4").tobytes()
    return n + payload + n


def read_records(data):
    """Split a sequential file into its record payloads."""
    out, p = [], 0
    while p < len(data):
        n = int(np.frombuffer(data[p:p + 4], "<i4")[0])
        payload = data[p + 4:p + 4 + n]
        m = int(np.frombuffer(data[p + 4 + n:p + 8 + n], "<i4")[0])
        assert m == n, "record markers disagree"
        out.append(payload)
        p += 8 + n
    return out


def f32(a):
    return np.ascontiguousarray(a, dtype="<f4").tobytes()


def me_of(turbulence):
    return 5 if turbulence else 4


def solu_written(q, qn, nut, turbulence):
    """The bytes output_restart writes (src/main.F90:346-370): one record each
    of q(m), m = 1..me; then nu_t when turbulent; then qn(m)."""
    q, qn = np.asarray(q).reshape(-1, 5), np.asarray(qn).reshape(-1, 5)
    me = me_of(turbulence)
    out = b"".join(record(f32(q[:, m])) for m in range(me))
    if turbulence:
        out += record(f32(nut))
    out += b"".join(record(f32(qn[:, m])) for m in range(me))
    return out


def solu_as_read(q, qn, nut, turbulence):
    """A file in the layout init_solu reads (src/init.F90:2392-2475): when
    turbulent, the records above; when laminar, q(1..me) as one record of
    me * N values (component-major), then qn likewise."""
    if turbulence:
        return solu_written(q, qn, nut, turbulence)
    q, qn = np.asarray(q).reshape(-1, 5), np.asarray(qn).reshape(-1, 5)
    me = me_of(turbulence)
    return record(f32(q[:, :me].T)) + record(f32(qn[:, :me].T))


def grid_bytes(x, y, z, wd, turbulence):
    """The grid file (src/init.F90:2226-2243): records x, y, z and, when
    turbulent, the wall distance."""
    arrs = [x, y, z] + ([wd] if turbulence else [])
    return b"".join(record(f32(a)) for a in arrs)


def filestat_read(text, n_tur):
    """time, step and turbine angles as src/init.F90:268-276 reads them; an
    angle >= 2 pi comes back by 2 pi."""
    tok = text.split()
    time, ntime = float(tok[0]), int(tok[1])
    ang = [float(t) for t in tok[2:2 + n_tur]]
    ang = [a - 2 * np.pi if a >= 2 * np.pi else a for a in ang]
    return time, ntime, ang
