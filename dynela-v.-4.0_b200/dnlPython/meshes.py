"""Mesh and model generators for the workloads the engine is measured on.

Units follow the DynELA samples: mm, s, tonne, MPa (Samples/Taylor/Taylor-Axi/Taylor.py:22-34).
Every generator returns a :class:`~dnlPython._abi.ModelDesc`; node and element
numbers are 0-based and ordered so that consecutive elements share nodes
(layer by layer along the bar axis), which keeps the nodal gathers local.
"""
import numpy as np

from . import _abi

# Copper (Taylor impact of the measured workloads): rho 8930 kg/m3, E 124 GPa,
# nu 0.34, Johnson-Cook A 90 MPa, B 292 MPa, n 0.31, C 0.025, eps0_dot 1/s,
# m 1.09, T0 298 K, Tm 1356 K, Cp 383 J/kgK, Taylor-Quinney 0.9.
COPPER = _abi.material(young=124000.0, poisson=0.34, density=8.93e-9, heat_capacity=3.83e8,
                       taylor_quinney=0.9, T0=298.0, A=90.0, B=292.0, C=0.025, n=0.31, m=1.09,
                       depsp0=1.0, Tm=1356.0, Tref=298.0)

# 42CrMo4 steel of the DynELA Taylor and necking samples (Taylor-Axi/Taylor.py:22-34).
STEEL_42CRMO4 = _abi.material(young=206000.0, poisson=0.3, density=7.83e-9, heat_capacity=4.6e8,
                              taylor_quinney=0.9, T0=20.0, A=806.0, B=614.0, C=0.0089, n=0.168, m=1.1,
                              depsp0=1.0, Tm=1540.0, Tref=20.0)

# Steel of the bar/plate necking workloads: rho 7800 kg/m3, E 206.9 GPa, nu 0.29,
# Johnson-Cook A 806, B 614, n 0.168, C 0.0089, m 1.1, Tm 1540 K, Cp 477 J/kgK.
STEEL_NECKING = _abi.material(young=206900.0, poisson=0.29, density=7.8e-9, heat_capacity=4.77e8,
                              taylor_quinney=0.9, T0=20.0, A=806.0, B=614.0, C=0.0089, n=0.168, m=1.1,
                              depsp0=1.0, Tm=1540.0, Tref=20.0)


def taylor_axi(nr=10, nz=80, radius=3.2, length=32.4, speed=227000.0, mat=COPPER, t_end=80e-6,
               ts_method=_abi.TS_COURANT, ts_freq=10, precision=_abi.PREC_FP64):
    """Axisymmetric Taylor bar of nr x nz ElQua4NAx elements, numbered as in
    Samples/Taylor/Taylor-Axi/Taylor.py:43-66 (rows of nr+1 nodes from the impact
    face up).  Impact face restrained axially, axis restrained radially,
    initial speed -speed along y."""
    dx, dy = radius / nr, length / nz
    j, i = np.meshgrid(np.arange(nz + 1), np.arange(nr + 1), indexing="ij")
    coords = np.zeros(((nr + 1) * (nz + 1), 3))
    coords[:, 0] = (i * dx).ravel()
    coords[:, 1] = (j * dy).ravel()
    jj, ii = np.meshgrid(np.arange(nz), np.arange(nr), indexing="ij")
    n1 = (ii + jj * (nr + 1)).ravel()
    conn = np.stack([n1, n1 + 1, n1 + nr + 2, n1 + nr + 1], axis=1)
    nN = coords.shape[0]
    bc = np.zeros((nN, 3), np.int8)
    bottom = coords[:, 1] == 0.0
    axis = coords[:, 0] == 0.0
    bc[bottom, 1] = _abi.BC_RESTRAIN
    bc[axis, 0] = _abi.BC_RESTRAIN
    v = np.zeros((nN, 3))
    v[:, 1] = -speed
    return _abi.ModelDesc(_abi.ELQUA4NAX, coords, conn, [mat], v_init=v, bc_code=bc, t_end=t_end,
                          ts_method=ts_method, ts_freq=ts_freq, precision=precision)


def _fix_hex_orientation(coords, conn):
    """Reverse the top/bottom faces of elements whose reference Jacobian is negative."""
    x = coords[conn]  # (nE, 8, 3)
    d1 = (x[:, 1] + x[:, 2] + x[:, 6] + x[:, 5]) - (x[:, 0] + x[:, 3] + x[:, 7] + x[:, 4])
    d2 = (x[:, 3] + x[:, 2] + x[:, 6] + x[:, 7]) - (x[:, 0] + x[:, 1] + x[:, 5] + x[:, 4])
    d3 = (x[:, 4] + x[:, 5] + x[:, 6] + x[:, 7]) - (x[:, 0] + x[:, 1] + x[:, 2] + x[:, 3])
    det = np.einsum("ij,ij->i", d1, np.cross(d2, d3))
    bad = det < 0
    conn = conn.copy()
    conn[bad] = conn[bad][:, [4, 5, 6, 7, 0, 1, 2, 3]]
    return conn


def _extrude(points2d, quads, nlayers, length, axis_offsets=None):
    """Extrude a cross-section in the (x, z) plane along y into hex8 elements."""
    nq = points2d.shape[0]
    ys = np.linspace(0.0, length, nlayers + 1) if axis_offsets is None else axis_offsets
    coords = np.zeros(((nlayers + 1) * nq, 3))
    for k, y in enumerate(ys):
        coords[k * nq:(k + 1) * nq, 0] = points2d[:, 0]
        coords[k * nq:(k + 1) * nq, 1] = y
        coords[k * nq:(k + 1) * nq, 2] = points2d[:, 1]
    conn = []
    for k in range(nlayers):
        b = quads + k * nq
        t = quads + (k + 1) * nq
        conn.append(np.concatenate([b, t], axis=1))
    conn = np.concatenate(conn, axis=0)
    return coords, _fix_hex_orientation(coords, conn)


def ogrid_section(radius, n_core, n_ring, core_frac=0.45):
    """O-grid disc: an n_core x n_core square core of half-width core_frac*radius
    and a ring of 4*n_core x n_ring quads blending the square's perimeter into
    the circle."""
    c = core_frac * radius  # half-width of the square core
    s = np.linspace(-c, c, n_core + 1)
    gx, gz = np.meshgrid(s, s, indexing="ij")
    core = np.stack([gx.ravel(), gz.ravel()], axis=1)
    idx = np.arange((n_core + 1) ** 2).reshape(n_core + 1, n_core + 1)
    quads = []
    for a in range(n_core):
        for b in range(n_core):
            quads.append([idx[a, b], idx[a + 1, b], idx[a + 1, b + 1], idx[a, b + 1]])
    # perimeter of the core, counter-clockwise, starting at corner (-c, -c)
    per = []
    n = n_core
    per += [idx[a, 0] for a in range(0, n)]          # bottom edge, x increasing
    per += [idx[n, b] for b in range(0, n)]          # right edge, z increasing
    per += [idx[a, n] for a in range(n, 0, -1)]      # top edge, x decreasing
    per += [idx[0, b] for b in range(n, 0, -1)]      # left edge, z decreasing
    per = np.array(per)
    nper = per.shape[0]
    theta = -0.75 * np.pi + 2.0 * np.pi * np.arange(nper) / nper
    circle = radius * np.stack([np.cos(theta), np.sin(theta)], axis=1)
    pts = [core]
    layer_ids = [per]
    nxt = core.shape[0]
    for l in range(1, n_ring + 1):
        t = l / n_ring
        p = (1.0 - t) * core[per] + t * circle
        pts.append(p)
        layer_ids.append(np.arange(nxt, nxt + nper))
        nxt += nper
    for l in range(n_ring):
        a, b = layer_ids[l], layer_ids[l + 1]
        for k in range(nper):
            k1 = (k + 1) % nper
            quads.append([a[k], a[k1], b[k1], b[k]])
    return np.concatenate(pts, axis=0), np.array(quads, dtype=np.int64)


def taylor_3d(n_core=12, n_ring=17, n_axial=160, radius=3.2, length=32.4, speed=227000.0, mat=COPPER,
              t_end=80e-6, ts_method=_abi.TS_COURANT, ts_freq=10, precision=_abi.PREC_MIXED):
    """Full 3-D Taylor bar on ElHex8N3D: an O-grid cross-section of
    n_core^2 + 4*n_core*n_ring quads extruded in n_axial layers along y.
    Defaults give 960 x 160 = 153,600 elements.  Impact face (y = 0) restrained
    along y, initial speed -speed along y."""
    pts, quads = ogrid_section(radius, n_core, n_ring)
    coords, conn = _extrude(pts, quads, n_axial, length)
    nN = coords.shape[0]
    bc = np.zeros((nN, 3), np.int8)
    bc[coords[:, 1] == 0.0, 1] = _abi.BC_RESTRAIN
    v = np.zeros((nN, 3))
    v[:, 1] = -speed
    return _abi.ModelDesc(_abi.ELHEX8N3D, coords, conn, [mat], v_init=v, bc_code=bc, t_end=t_end,
                          ts_method=ts_method, ts_freq=ts_freq, precision=precision)


def hex_block(nx, ny, nz, size=(1.0, 1.0, 1.0), mat=COPPER, t_end=1e-6, speed=0.0, seed=None,
              distort=0.0, precision=_abi.PREC_FP64, ts_freq=10):
    """Structured block of nx*ny*nz ElHex8N3D (test fixture).  With a seed, the
    interior nodes are jittered by `distort` x the cell size and the initial
    speed field is random with magnitude ~speed."""
    xs = np.linspace(0, size[0], nx + 1)
    ys = np.linspace(0, size[1], ny + 1)
    zs = np.linspace(0, size[2], nz + 1)
    gx, gy, gz = np.meshgrid(xs, ys, zs, indexing="ij")
    coords = np.stack([gx.ravel(), gy.ravel(), gz.ravel()], axis=1)
    idx = np.arange(coords.shape[0]).reshape(nx + 1, ny + 1, nz + 1)
    conn = []
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                conn.append([idx[i, j, k], idx[i + 1, j, k], idx[i + 1, j + 1, k], idx[i, j + 1, k],
                             idx[i, j, k + 1], idx[i + 1, j, k + 1], idx[i + 1, j + 1, k + 1], idx[i, j + 1, k + 1]])
    conn = np.array(conn)
    rng = np.random.default_rng(seed)
    if seed is not None and distort > 0:
        h = min(size[0] / nx, size[1] / ny, size[2] / nz)
        coords = coords + distort * h * rng.uniform(-1, 1, coords.shape)
    v = np.zeros_like(coords)
    if speed:
        if seed is None:
            v[:, 1] = -speed
        else:
            v = speed * rng.uniform(-1, 1, coords.shape)
    bc = np.zeros(coords.shape, np.int8)
    bc[coords[:, 1] <= 1e-12, 1] = _abi.BC_RESTRAIN
    conn = _fix_hex_orientation(coords, conn)
    return _abi.ModelDesc(_abi.ELHEX8N3D, coords, conn, [mat], v_init=v, bc_code=bc, t_end=t_end,
                          precision=precision, ts_freq=ts_freq)


def nodes_per_element_ratio(desc):
    return desc.n_nodes / desc.n_elems


def taylor_batch(n=256, seed=20261203, elems=(2000, 60000), speed=(150000.0, 300000.0), jc_scale=(0.8, 1.2),
                 t_end=80e-6, precision=_abi.PREC_MIXED, ts_freq=10):
    """Batch of independent 3-D copper Taylor bars of uneven size and parameters:
    element counts log-uniform in `elems`, impact speed uniform in `speed`
    (mm/s), and Johnson-Cook A, B, n, C, m each scaled by a factor uniform in
    `jc_scale`, all drawn from `seed`.  Each bar is taylor_3d with its
    cross-section and layer count scaled so that the elements keep the shape
    of the 153,600-element bar."""
    rng = np.random.default_rng(seed)
    descs = []
    for _ in range(n):
        target = float(np.exp(rng.uniform(np.log(elems[0]), np.log(elems[1]))))
        v = float(rng.uniform(*speed))
        f = rng.uniform(jc_scale[0], jc_scale[1], 5)
        mat = dict(COPPER)
        for k, s in zip(("A", "B", "n", "C", "m"), f):
            mat[k] = COPPER[k] * float(s)
        s = (target / 153600.0) ** (1.0 / 3.0)
        n_core = max(2, int(round(12 * s)))
        n_ring = max(2, int(round(17 * s)))
        per_layer = n_core * n_core + 4 * n_core * n_ring
        n_axial = max(4, int(round(target / per_layer)))
        descs.append(taylor_3d(n_core=n_core, n_ring=n_ring, n_axial=n_axial, speed=v, mat=mat, t_end=t_end,
                               ts_freq=ts_freq, precision=precision))
    return descs


def _pull_end(coords, length, speed, t_end, ramp_frac):
    """Symmetry plane y = 0 restrained along y; the end y = length pulled at
    `speed` along y, ramped linearly from 0 over the first ramp_frac of the run
    (a DiscreteFunction on the imposed speed, Boundary::setFunction)."""
    nN = coords.shape[0]
    bc = np.zeros((nN, 3), np.int8)
    val = np.zeros((nN, 3))
    fun = -np.ones((nN, 3), np.int32)
    bc[coords[:, 1] <= 1e-9, 1] = _abi.BC_RESTRAIN
    top = coords[:, 1] >= length - 1e-9
    bc[top, 1] = _abi.BC_SPEED
    val[top, 1] = speed
    fun[top, 1] = 0
    ramp = (np.array([0.0, ramp_frac * t_end, 2.0 * t_end]), np.array([0.0, 1.0, 1.0]))
    return dict(bc_code=bc, bc_value=val, bc_func=fun, functions=[ramp], v_init=np.zeros((nN, 3)))


def necking_end_time(elongation, speed, ramp_frac):
    """Time at which an end pulled at `speed`, ramped over the first ramp_frac
    of the run, has moved by `elongation`."""
    return elongation / (speed * (1.0 - 0.5 * ramp_frac))


def bar_necking(n_core=24, n_ring=34, n_axial=312, radius=6.413, length=26.667, reduction=0.01, speed=5000.0,
                elongation=7.0, ramp_frac=0.1, mat=STEEL_NECKING, precision=_abi.PREC_MIXED, ts_freq=10):
    """Round bar in tension, half of it (y >= 0, symmetry plane y = 0): an
    O-grid cross-section extruded along y, the radius reduced by `reduction`
    at y = 0 and tapered back to `radius` at y = length / 3 (the notch zone of
    Samples/BarNecking/BarNecking-3D/BarNecking.py).  The end is pulled at
    `speed` (mm/s), ramped over the first ramp_frac of the run, up to
    `elongation` mm.  Defaults: 3,840 x 312 = 1,198,080 elements."""
    pts, quads = ogrid_section(1.0, n_core, n_ring)
    coords, conn = _extrude(pts, quads, n_axial, length)
    zone = length / 3.0
    r = radius * (1.0 - reduction * np.clip(1.0 - coords[:, 1] / zone, 0.0, 1.0))
    coords[:, 0] *= r
    coords[:, 2] *= r
    t_end = necking_end_time(elongation, speed, ramp_frac)
    return _abi.ModelDesc(_abi.ELHEX8N3D, coords, conn, [mat], t_end=t_end, ts_freq=ts_freq, precision=precision,
                          **_pull_end(coords, length, speed, t_end, ramp_frac))


def _block(nx, ny, nz, x0, x1, y0, y1, z0, z1):
    """Structured hex8 block (vectorised), nodes x fastest then z then y
    (layer by layer along y)."""
    xs, ys, zs = np.linspace(x0, x1, nx + 1), np.linspace(y0, y1, ny + 1), np.linspace(z0, z1, nz + 1)
    gy, gz, gx = np.meshgrid(ys, zs, xs, indexing="ij")
    coords = np.stack([gx.ravel(), gy.ravel(), gz.ravel()], axis=1)
    idx = np.arange(coords.shape[0]).reshape(ny + 1, nz + 1, nx + 1)
    j, k, i = np.meshgrid(np.arange(ny), np.arange(nz), np.arange(nx), indexing="ij")
    j, k, i = j.ravel(), k.ravel(), i.ravel()
    conn = np.stack([idx[j, k, i], idx[j, k, i + 1], idx[j, k + 1, i + 1], idx[j, k + 1, i],
                     idx[j + 1, k, i], idx[j + 1, k, i + 1], idx[j + 1, k + 1, i + 1], idx[j + 1, k + 1, i]], axis=1)
    return coords, _fix_hex_orientation(coords, conn)


def plate_necking(nx=128, nz=12, ny=320, width=10.0, thickness=1.0, length=25.0, reduction=0.01, speed=5000.0,
                  elongation=7.0, ramp_frac=0.1, mat=STEEL_NECKING, precision=_abi.PREC_MIXED, ts_freq=10):
    """Flat plate in tension, half of it (y >= 0, symmetry plane y = 0),
    width x thickness cross-section centred on the y axis, the width reduced
    by `reduction` at y = 0 and tapered back at y = length / 3; end pulled as
    in bar_necking.  Defaults: 128 x 12 x 320 = 491,520 elements."""
    coords, conn = _block(nx, ny, nz, -0.5 * width, 0.5 * width, 0.0, length, -0.5 * thickness, 0.5 * thickness)
    zone = length / 3.0
    coords[:, 0] *= 1.0 - reduction * np.clip(1.0 - coords[:, 1] / zone, 0.0, 1.0)
    t_end = necking_end_time(elongation, speed, ramp_frac)
    return _abi.ModelDesc(_abi.ELHEX8N3D, coords, conn, [mat], t_end=t_end, ts_freq=ts_freq, precision=precision,
                          **_pull_end(coords, length, speed, t_end, ramp_frac))


def quad_block(nx, ny, size=(1.0, 1.0), mat=COPPER, t_end=1e-6, speed=0.0, seed=None, distort=0.0,
               precision=_abi.PREC_FP64, ts_freq=10, elem_type=_abi.ELQUA4N2D):
    """Structured block of nx*ny 4-node quads in the (x, y) plane (plane strain
    by default; elem_type=ELQUA4NAX for the axisymmetric element), nodes
    numbered row by row from y = 0.  With a seed, interior nodes are jittered by
    `distort` x the cell size and the initial speed is random with magnitude
    ~speed; y = 0 is restrained along y."""
    xs, ys = np.linspace(0, size[0], nx + 1), np.linspace(0, size[1], ny + 1)
    gy, gx = np.meshgrid(ys, xs, indexing="ij")
    coords = np.zeros(((nx + 1) * (ny + 1), 3))
    coords[:, 0], coords[:, 1] = gx.ravel(), gy.ravel()
    jj, ii = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    n1 = (ii + jj * (nx + 1)).ravel()
    conn = np.stack([n1, n1 + 1, n1 + nx + 2, n1 + nx + 1], axis=1)
    rng = np.random.default_rng(seed)
    if seed is not None and distort > 0:
        h = min(size[0] / nx, size[1] / ny)
        inner = (coords[:, 0] > 0) & (coords[:, 0] < size[0]) & (coords[:, 1] > 0) & (coords[:, 1] < size[1])
        coords[inner, :2] += distort * h * rng.uniform(-1, 1, (inner.sum(), 2))
    v = np.zeros_like(coords)
    if speed:
        v[:, :2] = speed * rng.uniform(-1, 1, (coords.shape[0], 2)) if seed is not None else [0.0, -speed]
    bc = np.zeros(coords.shape, np.int8)
    bc[coords[:, 1] <= 1e-12, 1] = _abi.BC_RESTRAIN
    return _abi.ModelDesc(elem_type, coords, conn, [mat], v_init=v, bc_code=bc, t_end=t_end, precision=precision,
                          ts_freq=ts_freq)
