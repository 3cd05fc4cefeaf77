"""Seeded synthetic cases with the shapes of the reference workloads.

The reference ships no grids or solutions ('grid', 'solu' files are read at
src/init.F90:2226-2243,2392-2411 but none are included), so every workload is
generated here from numpy's default_rng(seed).  Each builder returns
(case, grid, state) where grid = dict(x, y, z, wd) with arrays x(i,j,k)
(i fastest, Fortran order) and state = dict(q, qn, qnm1, nut) with q(1:5,i,j,k).

Presets
  cavity   laminar lid-driven cavity, Re = 1000, unit cube with interior nodes
           displaced by a seeded sinusoid of amplitude 0.02 h, 3-level FAS.
  channel  SA RANS channel at Re_tau = 395: tanh wall-normal stretching (first
           cell y+ ~ 1), nu_tilde = 3 nu, periodic i/k faces.
  ogrid    O-grid around a circular cylinder (radial geometric stretching to
           20 D, span pi D), SA, Re = 3900, delti = 0.005.
  wake     open box with uniform inflow and the characteristics outlet
           (btype 5), stretched and perturbed grid, SA or laminar.
  turbine  actuator-line turbine box 10 D x 5 D x 5 D (385 x 193 x 193), a
           3-blade rotor, TSR 7, eps = 0.05 D, inflow, outlet, SA.
"""
import numpy as np

from .abi import Case, BC_WALL, BC_SYMMETRY, BC_INFLOW, BC_OUTLET, BC_PERIODIC, BC_FREESTREAM, FP64, PRED_QN


def _base_case(im, jm, km):
    c = Case()
    c.im, c.jm, c.km = im, jm, km
    c.ng = 3
    c.icrs = c.jcrs = c.kcrs = 1
    for n, v in enumerate((1, 2, 3, 3)):
        c.iter[n] = v
    c.itmax = 200
    c.it_min = 7
    c.er_min = -6.0
    c.eo_min = -14.0
    c.delti = 0.05
    c.ren = 1000.0
    c.beta = 1.0
    c.cfl1, c.vnn1 = 1.0, 0.1
    c.cfl2, c.vnn2 = 0.5, 0.05
    c.itk = 2
    for d, v in enumerate((1.0, 2.5, 2.5)):
        c.ep[0][d] = v
    for d, v in enumerate((0.1, 0.2, 0.2)):
        c.ep[1][d] = v
    c.pdiss_coef = 0.1
    for b in range(6):
        c.btype[b] = BC_WALL
    for b, v in enumerate((1, 1, 2, 2, 3, 3)):
        c.bdir[b] = v
    c.ifix = c.jfix = c.kfix = 1
    c.turbulence = 0
    c.unsteady = 1
    c.conservation = 0
    c.precision_mode = FP64
    c.predictor = PRED_QN
    c.use_graph = 0
    return c


def _mesh(xs, ys, zs):
    """Fortran-order (i fastest) flattened coordinate arrays of a product grid."""
    X = np.empty((len(zs), len(ys), len(xs)))
    Y = np.empty_like(X)
    Z = np.empty_like(X)
    X[:] = xs[None, None, :]
    Y[:] = ys[None, :, None]
    Z[:] = zs[:, None, None]
    return X, Y, Z


def _flat(a):
    return np.ascontiguousarray(a.reshape(-1), dtype=np.float64)


def cavity(n=65, seed=0, re=1000.0, amp=0.02, ng=3, itmax=200):
    """Lid-driven cavity on a perturbed unit cube (wall faces, lid at j = jm).

    The lid is a btype-4 face holding u = 1 (bcond_fm only re-extrapolates the
    pressure there, src/bcond_fm.F90:221-229); the other five faces are
    no-slip walls.  Interior nodes move by amp * h * s(x,y,z) with s a product
    of sines with seeded phases that vanishes on every face.
    """
    rng = np.random.default_rng(seed)
    c = _base_case(n, n, n)
    c.ng = ng
    c.ren = re
    c.itmax = itmax
    c.btype[3] = BC_INFLOW
    h = 1.0 / (n - 1)
    s = np.linspace(0.0, 1.0, n)
    X, Y, Z = _mesh(s, s, s)
    bump = np.sin(np.pi * X) * np.sin(np.pi * Y) * np.sin(np.pi * Z)
    ph = rng.uniform(0, 2 * np.pi, size=(3, 3))
    wv = rng.integers(1, 4, size=(3, 3))
    disp = []
    for a in range(3):
        w = (np.sin(wv[a, 0] * 2 * np.pi * X + ph[a, 0]) *
             np.sin(wv[a, 1] * 2 * np.pi * Y + ph[a, 1]) *
             np.sin(wv[a, 2] * 2 * np.pi * Z + ph[a, 2]))
        disp.append(amp * h * bump * w)
    X = X + disp[0]
    Y = Y + disp[1]
    Z = Z + disp[2]
    grid = dict(x=_flat(X), y=_flat(Y), z=_flat(Z), wd=None)
    N = n ** 3
    q = np.zeros((N, 5))
    q[:, 1:4] = rng.normal(0.0, 1e-3, size=(N, 3))
    q = q.reshape(n, n, n, 5)          # [k][j][i][m]
    # walls: zero velocity; lid (j = jm): u = 1, v = w = 0
    for sl in [(slice(None), slice(None), 0), (slice(None), slice(None), -1),
               (slice(None), 0, slice(None)), (0, slice(None), slice(None)),
               (-1, slice(None), slice(None))]:
        q[sl + (slice(1, 4),)] = 0.0
    q[:, -1, :, 1] = 1.0
    q[:, -1, :, 2:4] = 0.0
    q = q.reshape(-1)
    state = dict(q=q.copy(), qn=q.copy(), qnm1=q.copy(), nut=np.zeros(N))
    return c, grid, state


def _tanh_stretch(jm, first, length=2.0):
    """Symmetric tanh clustering on [0, length] with first spacing ~ first."""
    eta = np.linspace(0.0, 1.0, jm)

    def ys(g):
        return 0.5 * length * (1.0 - np.tanh(g * (1.0 - 2.0 * eta)) / np.tanh(g))

    lo, hi = 1e-3, 10.0
    for _ in range(200):
        g = 0.5 * (lo + hi)
        if ys(g)[1] > first:
            lo = g
        else:
            hi = g
    return ys(0.5 * (lo + hi))


def _sa_fv1(nut_tilde, ren):
    chi = nut_tilde * ren
    chic = chi ** 3
    return nut_tilde * chic / (chic + 357.911)


def channel(im=129, jm=97, km=65, seed=0, re_tau=395.0, itmax=400, wall_first=None):
    """SA channel: i streamwise (2 pi), j wall-normal (walls at j = 1, jm),
    k spanwise (pi); half height 1, bulk velocity ~ 1.  Re based on the half
    height and bulk velocity (6875 for Re_tau = 395, Dean's correlation).
    The first wall spacing is 1 / Re_tau (y+ ~ 1) unless wall_first gives it
    (a coarse wall spacing, for the wall functions)."""
    rng = np.random.default_rng(seed)
    c = _base_case(im, jm, km)
    re_b = 2.0 * (re_tau / 0.09) ** (1.0 / 0.88)   # Re_bulk on 2 delta
    c.ren = 0.5 * re_b
    c.turbulence = 1
    c.itmax = itmax
    c.delti = 0.02
    c.btype[0] = c.btype[1] = BC_PERIODIC
    c.btype[2] = c.btype[3] = BC_WALL
    c.btype[4] = c.btype[5] = BC_PERIODIC
    c.ifix, c.jfix, c.kfix = im // 2, jm // 2, km // 2
    xs = np.linspace(0.0, 2 * np.pi, im)
    zs = np.linspace(0.0, np.pi, km)
    ys = _tanh_stretch(jm, wall_first if wall_first else 1.0 / re_tau)
    X, Y, Z = _mesh(xs, ys, zs)
    wd = np.minimum(Y, 2.0 - Y)
    grid = dict(x=_flat(X), y=_flat(Y), z=_flat(Z), wd=_flat(wd))
    N = im * jm * km
    # mean profile: 1/7 power law with bulk ~ 1, plus seeded noise
    u = (8.0 / 7.0) * np.clip(wd, 0.0, 1.0) ** (1.0 / 7.0)
    q = np.zeros((km, jm, im, 5))
    q[..., 1] = u
    q[..., 1:4] += rng.normal(0.0, 1e-3, size=(km, jm, im, 3)) * (wd > 0)[..., None]
    q[:, 0, :, 1:4] = 0.0
    q[:, -1, :, 1:4] = 0.0
    nu = 1.0 / c.ren
    q[..., 4] = 3.0 * nu
    q[:, 0, :, 4] = 1e-7
    q[:, -1, :, 4] = 1e-7
    q = q.reshape(-1)
    nut = _sa_fv1(q[4::5], c.ren)
    state = dict(q=q.copy(), qn=q.copy(), qnm1=q.copy(), nut=nut)
    return c, grid, state


def ogrid(im=257, jm=129, km=65, seed=0, re=3900.0, rfar=20.0, itmax=400):
    """O-grid around a unit-diameter cylinder: i azimuthal (periodic faces),
    j radial from the wall (j = 1) to a free-stream face at rfar diameters,
    k spanwise over pi D; SA with nu_tilde = 3 nu; uniform free stream plus
    seeded noise."""
    rng = np.random.default_rng(seed)
    c = _base_case(im, jm, km)
    c.ren = re
    c.turbulence = 1
    c.itmax = itmax
    c.delti = 0.005
    c.btype[0] = c.btype[1] = BC_PERIODIC
    c.btype[2] = BC_WALL
    c.btype[3] = BC_FREESTREAM
    c.btype[4] = c.btype[5] = BC_PERIODIC
    c.ifix, c.jfix, c.kfix = 1, jm, 1
    th = np.linspace(0.0, 2 * np.pi, im)
    r0 = 0.5
    first = 0.5 / np.sqrt(re) / 10.0
    lo, hi = 1.0 + 1e-9, 2.0
    for _ in range(200):  # geometric ratio with r(jm) = rfar
        g = 0.5 * (lo + hi)
        rend = r0 + first * (g ** (jm - 1) - 1.0) / (g - 1.0)
        if rend > rfar:
            hi = g
        else:
            lo = g
    g = 0.5 * (lo + hi)
    r = r0 + first * (g ** np.arange(jm) - 1.0) / (g - 1.0)
    zs = np.linspace(0.0, np.pi, km)
    TH = np.broadcast_to(th[None, None, :], (km, jm, im))
    RR = np.broadcast_to(r[None, :, None], (km, jm, im))
    ZZ = np.broadcast_to(zs[:, None, None], (km, jm, im))
    X = RR * np.cos(TH)
    Y = -RR * np.sin(TH)
    wd = RR - r0
    grid = dict(x=_flat(X), y=_flat(Y), z=_flat(ZZ), wd=_flat(wd))
    N = im * jm * km
    q = np.zeros((km, jm, im, 5))
    ramp = np.clip((RR - r0) / 1.0, 0.0, 1.0)
    q[..., 1] = ramp
    q[..., 1:4] += rng.normal(0.0, 1e-3, size=(km, jm, im, 3)) * (ramp > 0)[..., None]
    q[:, 0, :, 1:4] = 0.0
    q[..., 4] = 3.0 / c.ren
    q[:, 0, :, 4] = 1e-7
    q = q.reshape(-1)
    nut = _sa_fv1(q[4::5], c.ren)
    state = dict(q=q.copy(), qn=q.copy(), qnm1=q.copy(), nut=nut)
    return c, grid, state


def alm_rotor(xs, ys, zs, center, radius, nblades=3, nelems=12, nangles=24, tsr=7.0, hub_frac=0.1,
              length_scale=1.0, vel_infty=0.1, angle=0.3, seed=0, ker_cells=3, eps=None, narrow_polar=True):
    """Seeded synthetic actuator-line tables for one rotor on a product grid
    (coordinates xs[i], ys[j], zs[k]) with its plane normal to x, as the
    reference's init_lines places it (src/init.F90:1446-1535): element elem
    of azimuth bin nang sits at (xc, yc + r_e cos th, zc + r_e sin th) with
    r_e = radius elem / nelems and th = nang 2 pi / nangles.  Lengths are grid
    units except tur_rad and hub_rad (m = grid units x length_scale).  Three
    polars: wide, medium and one so narrow ([-2, 2] degrees) that many
    elements fall outside it (narrow_polar=False: a second wide one instead).
    The Gaussian width is the reference's eps = 2 dV^(1/3) of each kernel
    node (src/rhs_lines.F90:434); eps (grid units) fixes it instead: the
    kernel nodes are those within 3 eps of the rotor disc, and each carries
    dV = (eps / 2)^3, so that 2 dV^(1/3) = eps.  Returns the turbine dict and
    the polars."""
    rng = np.random.default_rng(seed)
    im, jm, km = len(xs), len(ys), len(zs)
    xc, yc, zc = center

    def cell(v, a, n):  # 1-based lower-corner index of the cell holding v
        return int(min(max(np.searchsorted(a, v, side="right"), 1), n - 1))

    node_index, node_pos = [], []
    dth = 2 * np.pi / nangles
    for nang in range(1, nangles + 1):
        th = nang * dth
        for elem in range(1, nelems + 1):
            x = xc
            y = yc + (radius / nelems) * elem * np.cos(th)
            z = zc + (radius / nelems) * elem * np.sin(th)
            i, j, k = cell(x, xs, im), cell(y, ys, jm), cell(z, zs, km)
            node_index.append((i, j, k))
            c = []
            for (a, b, d) in ((0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)):
                c += [xs[i - 1 + a], ys[j - 1 + b], zs[k - 1 + d]]
            node_pos.append([x, y, z] + c)
    J, K = np.meshgrid(np.arange(jm), np.arange(km), indexing="xy")  # [k][j]
    Y, Z = ys[J], zs[K]
    r = np.sqrt((Y - yc) ** 2 + (Z - zc) ** 2)
    dy = np.gradient(ys)[J]
    dz = np.gradient(zs)[K]
    dx = float(np.gradient(xs)[int(np.argmin(np.abs(xs - xc)))])
    rr = np.clip(r / radius, 0.0, 1.5)
    disk = np.zeros((km, jm, 8))
    disk[..., 0] = r
    disk[..., 1] = dy * dz
    disk[..., 2] = np.arctan2(Z - zc, Y - yc)
    disk[..., 3] = dx * dy * dz
    disk[..., 4] = 0.02 * (1.0 - 0.5 * rr)
    disk[..., 5] = 10.0 - 8.0 * rr + rng.normal(0.0, 0.5, size=r.shape)
    disk[..., 6] = rng.uniform(0.0, 1.0, size=r.shape)
    disk[..., 7] = 0.2
    polars = []
    spans = ((-30.0, 30.0, 25), (-12.0, 16.0, 15), (-2.0, 2.0, 5) if narrow_polar else (-90.0, 90.0, 37))
    for lo, hi, n in spans:
        a = np.linspace(lo, hi, n)
        cl = 2 * np.pi * np.deg2rad(a) * (1.0 + 0.05 * rng.normal(size=n))
        cd = 0.01 + 0.02 * (np.deg2rad(a)) ** 2 + 0.001 * rng.uniform(size=n)
        polars.append(np.vstack([np.column_stack([a, cl, cd]), [[-999.0, 0.0, 0.0]]]))
    pb = rng.integers(0, len(polars), size=(km, jm))
    pa = rng.integers(0, len(polars), size=(km, jm))
    h = max(dx, float(np.max(np.gradient(ys))), float(np.max(np.gradient(zs))))
    gx, gy, gz = np.gradient(xs), np.gradient(ys), np.gradient(zs)
    K3, J3, I3 = np.meshgrid(np.arange(2, km), np.arange(2, jm), np.arange(2, im), indexing="ij")
    X3, Y3, Z3 = xs[I3 - 1], ys[J3 - 1], zs[K3 - 1]
    R3 = np.hypot(Y3 - yc, Z3 - zc)
    if eps is None:
        sel = (np.abs(X3 - xc) <= ker_cells * dx) & (R3 <= radius + ker_cells * h)  # k, j, i order
        dV = (gx[I3 - 1] * gy[J3 - 1] * gz[K3 - 1])[sel]
    else:
        sel = (np.abs(X3 - xc) <= 3.0 * eps) & (R3 <= radius + 3.0 * eps)
        dV = np.full(int(sel.sum()), (0.5 * eps) ** 3)
    ker_index = np.column_stack([I3[sel], J3[sel], K3[sel]])
    ker_pos = np.column_stack([X3[sel], Y3[sel], Z3[sel]])
    ker_dat = np.column_stack([R3[sel], (gy[J3 - 1] * gz[K3 - 1])[sel], np.arctan2(Z3 - zc, Y3 - yc)[sel], dV])
    tur = dict(nblades=nblades, nelems=nelems, nangles=nangles, tsr=tsr,
               tur_rad=radius * length_scale, hub_rad=hub_frac * radius * length_scale, angle=angle,
               node_index=np.array(node_index, np.int32), node_pos=np.array(node_pos),
               disk_dat=disk.reshape(-1, 8), polar_b=pb.reshape(-1).astype(np.int32),
               polar_a=pa.reshape(-1).astype(np.int32),
               ker_index=np.array(ker_index, np.int32).reshape(-1, 3), ker_pos=np.array(ker_pos).reshape(-1, 3),
               ker_dat=np.array(ker_dat).reshape(-1, 4))
    return tur, polars


def wake(im=49, jm=25, km=25, seed=0, re=1000.0, turbulence=1, itmax=20, amp=0.05, side=BC_SYMMETRY, ng=3,
         noise=0.01):
    """Open box [0, 4] x [0, 2] x [0, 2] with a stream through it: uniform
    inflow u = 1 at i = 1 (btype 4: velocity held, pressure extrapolated with
    the grid ratio), the characteristics outlet at i = im (btype 5), 'side'
    on the j faces (symmetry planes by default) and periodic k faces.  x is
    stretched geometrically (ratio 1.02) so that the extrapolation ratios
    differ from 1; interior nodes and the outlet plane's y move by a seeded
    sinusoid, so that the outlet's csi metrics have cross components.  The
    state is the stream plus seeded noise of standard deviation 'noise'
    (velocity) and noise / 10 (pressure); nu_tilde = 3 nu and the wall
    distance is uniform (no walls) when turbulent."""
    rng = np.random.default_rng(seed)
    c = _base_case(im, jm, km)
    c.ng = ng
    c.ren = re
    c.itmax = itmax
    c.turbulence = turbulence
    c.btype[0], c.btype[1] = BC_INFLOW, BC_OUTLET
    c.btype[2] = c.btype[3] = side
    c.btype[4] = c.btype[5] = BC_PERIODIC
    g = 1.02 ** np.arange(im - 1)
    xs = np.concatenate(([0.0], np.cumsum(g))) * (4.0 / g.sum())
    ys = np.linspace(0.0, 2.0, jm)
    zs = np.linspace(0.0, 2.0, km)
    X, Y, Z = _mesh(xs, ys, zs)
    h = 2.0 / (jm - 1)
    ph = rng.uniform(0, 2 * np.pi, size=3)
    sy = np.sin(np.pi * Y / 2.0)
    sz = np.sin(np.pi * Z / 2.0)
    sx = np.sin(np.pi * X / 4.0)
    dx = amp * h * sx * sy * sz * np.cos(np.pi * Z + ph[0])
    dy = amp * h * (X / 4.0) * sy * sz * np.sin(np.pi * X + ph[1])
    dz = amp * h * sx * sy * sz * np.sin(np.pi * Y + ph[2])
    grid = dict(x=_flat(X + dx), y=_flat(Y + dy), z=_flat(Z + dz),
                wd=np.full(im * jm * km, 10.0) if turbulence else None)
    N = im * jm * km
    q = np.zeros((N, 5))
    q[:, 0] = rng.normal(0.0, 0.1 * noise, size=N)
    q[:, 1] = 1.0 + rng.normal(0.0, noise, size=N)
    q[:, 2:4] = rng.normal(0.0, noise, size=(N, 2))
    q = q.reshape(km, jm, im, 5)
    q[:, :, 0, 1] = 1.0               # inflow plane
    q[:, :, 0, 2:4] = 0.0
    if side == BC_SYMMETRY:
        q[:, 0, :, 2] = 0.0
        q[:, -1, :, 2] = 0.0
    nut = np.zeros(N)
    if turbulence:
        q[..., 4] = 3.0 / re
        nut[:] = _sa_fv1(q[..., 4].reshape(-1), re)
    q = q.reshape(-1)
    state = dict(q=q.copy(), qn=q.copy(), qnm1=q.copy(), nut=nut)
    return c, grid, state


def rfg_inflow(case, u=1.0, intensity=0.05, length_scale=0.2, time_scale=None, nmodes=1000, seed=0,
               tables=None):
    """Tables of the synthetic inflow turbulence (desalm_rfg) for the i = 1
    plane of 'case': mean velocity (u, 0, 0), an isotropic correlation tensor
    (intensity u)^2 I (the generator reproduces the tensor it is given: with
    k ~ N(0, 0.5^2) each unit mode pair has unit variance), length scale
    'length_scale', time scale 'time_scale' (default length_scale / u), and
    'nmodes' modes drawn by desalm_rfg_modes from 'seed' (or the given
    'tables': p, q, k, omega)."""
    jm, km = case.jm, case.km
    if tables is None:
        from .solver import rfg_modes
        tables = rfg_modes(nmodes, seed)
    um = np.zeros((km, jm, 3))
    um[..., 0] = u
    uij = np.zeros((km, jm, 6))
    uij[..., 0] = uij[..., 3] = uij[..., 5] = (intensity * u) ** 2
    ts = np.full((km, jm), length_scale / u if time_scale is None else time_scale)
    ls = np.full((km, jm), length_scale)
    return dict(tables, um=um, uij=uij, t_ts=ts, t_ls=ls)


def channel_alm(im=33, jm=25, km=25, itmax=20, n_tur=1, seed=0):
    """The SA channel with n_tur synthetic rotors (alm_rotor) along x; the
    Reynolds number gives vel_scale = ren 1e-6 / length_scale."""
    case, grid, state = channel(im=im, jm=jm, km=km, itmax=itmax, seed=seed)
    xs = np.linspace(0.0, 2 * np.pi, im)
    ys = _tanh_stretch(jm, 1.0 / 395.0)
    zs = np.linspace(0.0, np.pi, km)
    turs, polars = [], None
    for t in range(n_tur):
        xc = xs[int((t + 1) * im / (n_tur + 1))]
        tur, pol = alm_rotor(xs, ys, zs, (xc, 1.0, np.pi / 2), 0.5, seed=seed + t, angle=0.3 + 1.1 * t)
        turs.append(tur)
        polars = pol if polars is None else polars
    spec = dict(turbines=turs, polars=polars, vel_infty=0.1, length_scale=1.0)
    return case, grid, state, spec


def _sinh_cluster(n, length, centre, c):
    """n nodes on [0, length] clustered at x = centre: x = centre + B sinh(c (s - s0)),
    s uniform on [0, 1], s0 and B chosen so that the ends land on 0 and length."""
    s = np.linspace(0.0, 1.0, n)
    ratio = (length - centre) / centre
    lo, hi = 1e-6, 1.0 - 1e-6
    for _ in range(200):      # sinh(c (1 - s0)) / sinh(c s0) = ratio
        s0 = 0.5 * (lo + hi)
        if np.sinh(c * (1.0 - s0)) / np.sinh(c * s0) > ratio:
            lo = s0
        else:
            hi = s0
    s0 = 0.5 * (lo + hi)
    B = centre / np.sinh(c * s0)
    x = centre + B * np.sinh(c * (s - s0))
    x[0], x[-1] = 0.0, length
    return x


def turbine(im=385, jm=193, km=193, seed=0, re=1.0e5, itmax=400, delti=0.005, nelems=40, nangles=72,
            eps=0.05, stretch=2.0, ng=3, polar_seed=0):
    """Actuator-line turbine box: a 3-blade rotor of diameter D = 1 (the
    length unit) at (2.5, 2.5, 2.5) in a [0, 10] x [0, 5] x [0, 5] box
    (10 D x 5 D x 5 D), its plane normal to x; tip-speed ratio 7; Gaussian
    projection of width eps = 0.05 D; seeded synthetic polars (alm_rotor).
    The grid is a product of sinh-clustered lines (finest at the rotor,
    growing toward every face), uniform inflow u = 1 at i = 1 (btype 4), the
    characteristics outlet at i = im (btype 5) and symmetry planes on the
    j and k faces; SA with nu_tilde = 3 nu and no walls (wall distance 10).
    Velocities are scaled by vel_infty = Re 1e-6 / length_scale (0.1 m/s
    for Re_D = 1e5 and D = 1 m), so that the free stream is u = 1.
    Returns (case, grid, state, alm spec, omega), omega the rotor's angular
    speed in radians per unit of nondimensional time (D / U): the driver
    advances each azimuth by omega * delti between physical steps."""
    rng = np.random.default_rng(seed)
    c = _base_case(im, jm, km)
    c.ng = ng
    c.ren = re
    c.itmax = itmax
    c.delti = delti
    c.turbulence = 1
    c.btype[0], c.btype[1] = BC_INFLOW, BC_OUTLET
    c.btype[2] = c.btype[3] = BC_SYMMETRY
    c.btype[4] = c.btype[5] = BC_SYMMETRY
    c.ifix, c.jfix, c.kfix = im - 1, 2, 2
    xs = _sinh_cluster(im, 10.0, 2.5, stretch)
    ys = _sinh_cluster(jm, 5.0, 2.5, stretch)
    zs = _sinh_cluster(km, 5.0, 2.5, stretch)
    X, Y, Z = _mesh(xs, ys, zs)
    N = im * jm * km
    grid = dict(x=_flat(X), y=_flat(Y), z=_flat(Z), wd=np.full(N, 10.0))
    q = np.zeros((km, jm, im, 5))
    q[..., 1] = 1.0
    q[..., 1:4] += rng.normal(0.0, 1e-3, size=(km, jm, im, 3))
    q[:, :, 0, 1] = 1.0
    q[:, :, 0, 2:4] = 0.0
    q[:, 0, :, 2] = q[:, -1, :, 2] = 0.0
    q[0, :, :, 3] = q[-1, :, :, 3] = 0.0
    q[..., 4] = 3.0 / re
    q = q.reshape(-1)
    nut = _sa_fv1(q[4::5], re)
    state = dict(q=q.copy(), qn=q.copy(), qnm1=q.copy(), nut=nut)
    length_scale = 1.0
    vel = re * 1e-6 / length_scale
    tur, polars = alm_rotor(xs, ys, zs, (2.5, 2.5, 2.5), 0.5, nblades=3, nelems=nelems, nangles=nangles,
                            tsr=7.0, length_scale=length_scale, vel_infty=vel, angle=0.3, seed=polar_seed,
                            eps=eps, narrow_polar=False)
    spec = dict(turbines=[tur], polars=polars, vel_infty=vel, length_scale=length_scale)
    omega = 7.0 * 1.0 / 0.5          # TSR U / R in units of U / D
    return c, grid, state, spec, omega


def _host_cell(a, v):
    """Lower-corner index (0-based) and fraction of v in the sorted nodes a."""
    i = int(np.clip(np.searchsorted(a, v, side="right") - 1, 0, len(a) - 2))
    return i, (v - a[i]) / (a[i + 1] - a[i])


def overset_pair(seed=0, turbulence=1, itmax=20, re=1000.0):
    """Two overlapping wake boxes along x with trilinear donor maps: block 0
    spans x in [0, 2] (inflow at i = 1, an interface face at i = im), block 1
    x in [1.5, 3.5] (an interface face at i = 1, the characteristics outlet at
    i = im); both span y, z in [0, 2] but with different node counts, so the
    host cells of the interface nodes are interpolated in all three
    directions.  Each interface node (every j, k of the interface face) takes
    its values from the host cell of the other block that contains it.
    Returns ([(case, grid, state)] for the two blocks, map) with the map as
    desalm_overset_map arrays (0-based blocks, 1-based nodes)."""
    return overset_chain(2, seed=seed, turbulence=turbulence, itmax=itmax, re=re)


_CHAIN_DIMS = [(33, 21, 17), (29, 17, 21), (25, 21, 17), (37, 17, 21)]   # odd at every coarsening of 3 levels


def overset_chain(nblocks=2, seed=0, turbulence=1, itmax=20, re=1000.0):
    """nblocks (2..4) overlapping wake boxes along x, block b spanning x in
    [1.5 b, 1.5 b + 2] and y, z in [0, 2] with its own node counts (odd
    blocks cosine-clustered in y): inflow at block 0's i = 1, the
    characteristics outlet at the last block's i = im, interface faces
    between neighbours.  Block b's i = im face takes its values from block
    b + 1, its i = 1 face from block b - 1 (the donees in that order, block
    by block).  Returns ([(case, grid, state)], map) as overset_pair."""
    assert 2 <= nblocks <= len(_CHAIN_DIMS)
    rng = np.random.default_rng(seed)
    dims = _CHAIN_DIMS[:nblocks]
    xr = [(1.5 * b, 1.5 * b + 2.0) for b in range(nblocks)]
    blocks, axes = [], []
    for b, (im, jm, km) in enumerate(dims):
        c, g, st = wake(im=im, jm=jm, km=km, seed=seed + b, turbulence=turbulence, itmax=itmax, amp=0.0, re=re)
        c.btype[0] = BC_INFLOW if b == 0 else 0
        c.btype[1] = BC_OUTLET if b == nblocks - 1 else 0
        gx = 1.03 ** np.arange(im - 1)
        xs = xr[b][0] + np.concatenate(([0.0], np.cumsum(gx))) * ((xr[b][1] - xr[b][0]) / gx.sum())
        ys = np.linspace(0.0, 2.0, jm) ** 1.0
        ys = 2.0 * (0.5 - 0.5 * np.cos(np.pi * np.linspace(0.0, 1.0, jm))) if b % 2 == 1 else ys
        zs = np.linspace(0.0, 2.0, km)
        X, Y, Z = _mesh(xs, ys, zs)
        g = dict(x=_flat(X), y=_flat(Y), z=_flat(Z), wd=g.get("wd"))
        q = st["q"].reshape(-1, 5)
        q[:, 1] = 1.0 + 0.05 * np.sin(np.pi * X.reshape(-1)) * np.cos(np.pi * Y.reshape(-1) / 2.0)
        q[:, 2] = 0.02 * rng.normal(size=q.shape[0])
        st = dict(q=q.reshape(-1).copy(), qn=q.reshape(-1).copy(), qnm1=q.reshape(-1).copy(), nut=st["nut"])
        blocks.append((c, g, st))
        axes.append((xs, ys, zs))
    donee, host, coef = [], [], []
    for b in range(nblocks):
        im, jm, km = dims[b]
        xs, ys, zs = axes[b]
        faces = []
        if b < nblocks - 1:
            faces.append((im, b + 1))
        if b > 0:
            faces.append((1, b - 1))
        for i, other in faces:
            ox, oy, oz = axes[other]
            for k in range(1, km + 1):
                for j in range(1, jm + 1):
                    ih, fx = _host_cell(ox, xs[i - 1])
                    jh, fy = _host_cell(oy, ys[j - 1])
                    kh, fz = _host_cell(oz, zs[k - 1])
                    donee.append((b, i, j, k))
                    host.append((other, ih + 1, jh + 1, kh + 1))
                    coef.append((fx, fy, fz))
    ov = dict(donee=np.array(donee, np.int32).reshape(-1), host=np.array(host, np.int32).reshape(-1),
              coef=np.array(coef, np.float64).reshape(-1), n=len(donee))
    return blocks, ov


def kw_coef_as(k, w, ren):
    """Wilcox's alpha* = (0.15 + Re_t) / (6 + Re_t), Re_t = Re k / omega
    (src/rhs_kw_coef.F90:47-49)."""
    rt = ren * k / w
    return (0.15 + rt) / (6.0 + rt)


def with_kw(case, grid, state, intensity=0.01, nut_ratio=3.0):
    """The same case with the k-omega model (turbulence = 2): k = 1.5 (I |u|)^2
    from the state's velocity magnitude (at least 1.5 I^2 x 1e-4 of the
    free-stream value), omega such that nu_t = As k / omega is nut_ratio
    times the molecular viscosity, and k = 0 with the wall value of omega
    60 / (Re 0.075 yd^2) on wall faces, as rhs_kw_bcond sets them.  Returns
    (case, grid, state, omega) where state's fifth component is k and omega
    = dict(omega, omega_n, omega_nm1)."""
    c = case.copy()
    c.turbulence = 2
    N = c.im * c.jm * c.km
    q = state["q"].reshape(N, 5).copy()
    speed = np.sqrt(q[:, 1] ** 2 + q[:, 2] ** 2 + q[:, 3] ** 2)
    k = np.maximum(1.5 * (intensity * speed) ** 2, 1.5 * intensity ** 2 * 1e-4)
    nu = 1.0 / c.ren
    As = 0.5084   # the fixed point of As(Re_t) with nu_t = 3 nu
    w = As * k / (nut_ratio * nu)
    wd = grid.get("wd")
    kk = k.reshape(c.km, c.jm, c.im)
    ww = w.reshape(c.km, c.jm, c.im)
    wdr = None if wd is None else wd.reshape(c.km, c.jm, c.im)
    srenp = 60.0 / c.ren / 0.075
    faces = [(slice(None), slice(None), 0, (slice(None), slice(None), 1)),
             (slice(None), slice(None), -1, (slice(None), slice(None), -2)),
             (slice(None), 0, slice(None), (slice(None), 1, slice(None))),
             (slice(None), -1, slice(None), (slice(None), -2, slice(None))),
             (0, slice(None), slice(None), (1, slice(None), slice(None))),
             (-1, slice(None), slice(None), (-2, slice(None), slice(None)))]
    for b, f in enumerate(faces):
        if c.btype[b] == BC_WALL and wdr is not None:
            sl = f[:3]
            kk[sl] = 0.0
            yd = np.maximum(wdr[f[3]], 1e-12)
            ww[sl] = srenp / yd / yd
    k = kk.reshape(-1)
    w = ww.reshape(-1)
    q[:, 4] = k
    nut = kw_coef_as(k, w, c.ren) * k / w
    st = dict(q=q.reshape(-1).copy(), qn=q.reshape(-1).copy(), qnm1=q.reshape(-1).copy(), nut=nut)
    om = dict(omega=w.copy(), omega_n=w.copy(), omega_nm1=w.copy())
    return c, grid, st, om


PRESETS = {"cavity": cavity, "channel": channel, "ogrid": ogrid, "wake": wake}
