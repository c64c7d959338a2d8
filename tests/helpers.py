"""Shared helpers of the test suite: model descriptions, seeded random states,
fixture (de)serialisation and comparison utilities."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "dynela-v.-4.0_b200")
ORACLE = os.path.join(ROOT, "oracle")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (PKG, ORACLE):
    if p not in sys.path:
        sys.path.insert(0, p)

from dnlPython import _abi, meshes  # noqa: E402

# tolerance stated for the element pass (internal forces and returned stresses)
# of the FP64 path against the FP64 oracle: 1e-6 relative
FP64_PASS_RTOL = 1e-6
# mixed path (FP32 element math and point state) against the FP64 oracle on one pass
MIXED_PASS_RTOL = 2e-4


def desc_to_npz(desc, prefix=""):
    out = {}
    out[prefix + "elem_type"] = np.array(desc.elem_type)
    out[prefix + "coords"] = desc.coords
    out[prefix + "conn"] = desc.conn
    keys = [f[0] for f in _abi.Material._fields_]
    out[prefix + "materials"] = np.array([[m[k] for k in keys] for m in desc.materials])
    for name in ("elem_mat", "v_init", "bc_code", "bc_value", "bc_func"):
        a = getattr(desc, name)
        if a is not None:
            out[prefix + name] = a
    if desc.functions:
        out[prefix + "func_x"] = np.concatenate([f[0] for f in desc.functions])
        out[prefix + "func_y"] = np.concatenate([f[1] for f in desc.functions])
        out[prefix + "func_n"] = np.array([len(f[0]) for f in desc.functions])
    out[prefix + "solver"] = np.array([desc.t_start, desc.t_end, desc.ts_method, desc.ts_freq, desc.ts_safety,
                                       desc.rho_b, desc.precision, desc.stress_method])
    return out


def desc_from_npz(z, prefix="", precision=None):
    keys = [f[0] for f in _abi.Material._fields_]
    mats = [dict(zip(keys, row)) for row in z[prefix + "materials"]]
    funcs = []
    if prefix + "func_n" in z:
        x, y, off = z[prefix + "func_x"], z[prefix + "func_y"], 0
        for n in z[prefix + "func_n"]:
            funcs.append((x[off:off + n], y[off:off + n]))
            off += n
    s = z[prefix + "solver"]
    opt = {k: z[prefix + k] for k in ("elem_mat", "v_init", "bc_code", "bc_value", "bc_func") if prefix + k in z}
    return _abi.ModelDesc(int(z[prefix + "elem_type"]), z[prefix + "coords"], z[prefix + "conn"], mats,
                          functions=funcs, t_start=s[0], t_end=s[1], ts_method=int(s[2]), ts_freq=int(s[3]),
                          ts_safety=s[4], rho_b=s[5],
                          precision=int(s[6]) if precision is None else precision,
                          stress_method=int(s[7]) if len(s) > 7 else _abi.STRESS_NEWTON, **opt)


def random_point_state(desc, ips, seed, stress_scale=200.0):
    """A seeded, physically plausible integration-point state on top of the
    initial one (keeps detJ0 and density): stresses around the yield stress,
    a mix of virgin and plastified points."""
    rng = np.random.default_rng(seed)
    n = desc.n_ips
    s = ips.copy()
    mat = desc.materials[0]
    s[0:6] = rng.normal(0.0, stress_scale, (6, n))
    if desc.elem_type == _abi.ELQUA4NAX:
        s[2] = s[4] = 0.0
    s[6:12] = rng.normal(0.0, 0.05, (6, n))
    s[12:18] = rng.normal(0.0, 0.03, (6, n))
    if desc.elem_type == _abi.ELQUA4NAX:
        s[8] = s[10] = s[14] = s[16] = 0.0
    plastic = rng.uniform(size=n) < 0.7
    epsp = np.where(plastic, rng.uniform(0.0, 0.6, n), 0.0)
    s[_abi.IP_EPSP] = epsp
    s[_abi.IP_DEPSP] = np.where(plastic, rng.uniform(0.0, 2e4, n), 0.0)
    s[_abi.IP_GAMMA] = np.where(plastic, rng.uniform(1e-6, 5e-4, n), 0.0)
    s[_abi.IP_GAMMA_CUM] = np.where(plastic, epsp * 1.2247, 0.0)
    s[_abi.IP_YIELD] = np.where(plastic, mat["A"] + mat["B"] * np.power(np.maximum(epsp, 1e-12), mat["n"]), 0.0)
    s[_abi.IP_T] = mat["T0"] + rng.uniform(0.0, 250.0, n)
    s[_abi.IP_PRESSURE] = 0.0
    s[_abi.IP_EINT] = rng.uniform(0.0, 1e5, n)
    s[_abi.IP_EINEL] = rng.uniform(0.0, 1e5, n)
    return s


def random_increment(desc, seed, strain=2e-3):
    """Seeded displacement increment (field0->u) giving strain increments ~strain."""
    rng = np.random.default_rng(seed)
    x = desc.coords
    h = (x.max(0) - x.min(0)).max() / max(desc.n_elems ** (1.0 / (2 if desc.elem_type == _abi.ELQUA4NAX else 3)), 1)
    u = strain * h * rng.normal(size=(desc.n_nodes, 3))
    u += rng.normal(size=3) * 1e-3  # rigid translation part
    if desc.elem_type == _abi.ELQUA4NAX:
        u[:, 2] = 0.0
    return u


def rel_err(a, b, axis=None):
    """max |a - b| / max |b| (per row when axis=1)."""
    a = np.asarray(a)
    b = np.asarray(b)
    if axis is None:
        return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)
    return np.abs(a - b).max(axis=axis) / np.maximum(np.abs(b).max(axis=axis), 1e-300)


def field_errors(ga, gb):
    """Relative error of each point-state component: tensor components are
    scaled by the largest component of their tensor (stress, strain, plastic
    strain), scalars by their own largest value."""
    ga, gb = np.asarray(ga), np.asarray(gb)
    err = np.abs(ga - gb).max(axis=1)
    scale = np.abs(gb).max(axis=1)
    for b in (0, 6, 12):
        scale[b:b + 6] = scale[b:b + 6].max()
    return err / np.maximum(scale, 1e-300)


def field_sums(a):
    """Per component (column) of a [n, k] field: signed sum, sum of magnitudes
    and largest magnitude over every row, FP64 ([3, k])."""
    a = np.asarray(a, dtype=np.float64)
    return np.stack([a.sum(0), np.abs(a).sum(0), np.abs(a).max(0)])


def mesh_digest(desc):
    """Digest of a model's coordinates and connectivity (a fixture records it
    so that a test knows it rebuilt the same mesh)."""
    import hashlib
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(desc.coords, dtype=np.float64).tobytes())
    h.update(np.ascontiguousarray(desc.conn, dtype=np.int32).tobytes())
    return h.hexdigest()


def entry_errors(a, b, scale, floor=1e-4):
    """Entry by entry: |a - b| / (|b| + floor * scale), the largest over the
    entries of each row (a [k, n] array of k components); `scale` is the
    component's largest magnitude over the whole field.  A bound tol on it
    reads |a - b| <= tol |b| for every entry above `floor` of its field's
    largest magnitude, and |a - b| <= tol * floor * scale below: values that
    are themselves at the rounding level of their field (shear components
    cancelling to 1e-8 of the stress, say) are held to that absolute level
    instead of being divided by themselves."""
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    scale = np.asarray(scale, dtype=np.float64).reshape(-1, 1)
    return (np.abs(a - b) / (np.abs(b) + floor * scale + 1e-300)).max(axis=1)


def group_scale(values, groups=()):
    """Per component, the largest of `values` over its group: components
    of one quantity (a nodal vector's 3, a point-state tensor's 6) share a
    scale, so that a component that is itself at the noise level of the
    quantity is measured against the quantity."""
    out = np.array(values, dtype=np.float64)
    for b, n in groups:
        out[b:b + n] = out[b:b + n].max()
    return out


NODE_GROUPS = ((0, 3),)
IP_GROUPS = ((0, 6), (6, 6), (12, 6))


def sums_errors(a_sums, b_sums, groups=()):
    """Whole-field checks from field_sums: the sums of magnitudes and the
    largest magnitudes relative to themselves, the signed sums relative to
    the sum of magnitudes (a signed sum may cancel); with `groups`, relative
    to their group's largest."""
    a, b = np.asarray(a_sums), np.asarray(b_sums)
    den = np.maximum(group_scale(b[1], groups), 1e-300)
    return np.concatenate([np.abs(a[0] - b[0]) / den, np.abs(a[1] - b[1]) / den,
                           np.abs(a[2] - b[2]) / np.maximum(group_scale(b[2], groups), 1e-300)])


FULL_NODE_FIELDS = (("coords", _abi.NODE_COORDS), ("disp", _abi.NODE_DISP), ("speed", _abi.NODE_SPEED),
                    ("u", _abi.NODE_U), ("accel", _abi.NODE_ACCEL), ("force", _abi.NODE_FORCE))
FULL_ENTRY_RTOL = 1e-6
FULL_SUMS_RTOL = 1e-9
# where the problem's conditioning puts the C restatement further than the
# bounds above from the reference, the engine may be this many times as far
FULL_NOISE_FACTOR = 4.0


def full_size_errors(m, z, prefix, source=""):
    """A model (engine or oracle: nodes(field), ips()) against a full-size
    fixture's checkpoint `prefix`: per field, the entry errors of its sampled
    entries per component (entry_errors, the floor against its group's
    largest magnitude) and the errors of its whole-field sums (sums_errors,
    by group).  source "" compares with the reference's values, "_orc" with
    the C restatement's stored beside them (its polar decomposition on
    C = F^T F, as the reference's), "_orh" with the restatement's whose
    polar decomposition is formed from H = F - I (as the engine's)."""
    nodes, ips = z["sample_nodes"], z["sample_ips"]
    out = {}
    for name, f in FULL_NODE_FIELDS:
        a = m.nodes(f)
        sums = z[f"{prefix}{name}{source}_sums"]
        scale = group_scale(z[f"{prefix}{name}_sums"][2], NODE_GROUPS)
        out[name] = (entry_errors(a[nodes].T, z[f"{prefix}{name}{source}"].T, scale),
                     sums_errors(field_sums(a), sums, NODE_GROUPS))
    ip = m.ips()
    sums = z[f"{prefix}ips{source}_sums"]
    scale = group_scale(z[f"{prefix}ips_sums"][2], IP_GROUPS)
    out["ips"] = (entry_errors(ip[:, ips], z[f"{prefix}ips{source}"], scale),
                  sums_errors(field_sums(ip.T), sums, IP_GROUPS))
    return out


def check_full_size(m, z, prefix, what, noise="o", source=""):
    """full_size_errors within their bounds, per component: FULL_ENTRY_RTOL
    and FULL_SUMS_RTOL, or FULL_NOISE_FACTOR times a distance measured the
    same way and stored in the fixture, where that is larger: noise "o", the
    C oracle's own distance to the reference (`*_onoise`, `*_osums`); "h",
    the same for the C oracle with its polar decomposition formed from
    H = F - I (`*_hnoise`, `*_hsums`); "p", that oracle's distance to itself
    run from coordinates moved by one unit in the last place (`*_pnoise`,
    `*_psums`: how far rounding alone carries two FP64 runs of the same
    algorithm apart); None, the fixed bounds only.
    Returns per field (largest entry error, largest sums error, largest
    entry error over its bound)."""
    worst = {}
    for name, (err, serr) in full_size_errors(m, z, prefix, source).items():
        eb, sb = np.full(err.size, FULL_ENTRY_RTOL), np.full(serr.size, FULL_SUMS_RTOL)
        if noise and f"{prefix}{name}_{noise}noise" in z:
            eb = np.maximum(eb, FULL_NOISE_FACTOR * z[f"{prefix}{name}_{noise}noise"])
            sb = np.maximum(sb, FULL_NOISE_FACTOR * z[f"{prefix}{name}_{noise}sums"])
        worst[name] = (float(err.max()), float(serr.max()), float((err / eb).max()))
        assert np.all(err <= eb), (what, name, err, eb)
        assert np.all(serr <= sb), (what, name, serr, sb)
    return worst


# model cases shared by the golden fixtures and the parity tests
def case_axi_small(precision=_abi.PREC_FP64):
    return meshes.taylor_axi(nr=5, nz=20, radius=3.2, length=8.1, speed=227000.0, t_end=4e-6, ts_freq=1,
                             precision=precision)


def case_hex_small(precision=_abi.PREC_FP64):
    return meshes.hex_block(3, 4, 3, size=(0.9, 1.2, 0.9), speed=60000.0, seed=11, distort=0.12, t_end=5e-6,
                            precision=precision, ts_freq=3)


def case_hex_speed(precision=_abi.PREC_FP64):
    """Hex block pulled at its top face by an imposed speed ramped by a
    piecewise-linear function, bottom face restrained (necking-like loading)."""
    d = meshes.hex_block(3, 5, 3, size=(0.9, 1.5, 0.9), mat=meshes.STEEL_NECKING, t_end=4e-6, precision=precision,
                         ts_freq=2)
    top = d.coords[:, 1] >= d.coords[:, 1].max() - 1e-12
    bc = d.bc_code.copy()
    val = np.zeros_like(d.coords)
    fun = -np.ones(d.coords.shape, np.int32)
    bc[top, 1] = _abi.BC_SPEED
    val[top, 1] = 5000.0
    fun[top, 1] = 0
    ramp = (np.array([0.0, 1e-6, 1.0]), np.array([0.0, 1.0, 1.0]))
    return d.copy(bc_code=bc, bc_value=val, bc_func=fun, functions=[ramp], v_init=np.zeros_like(d.coords))


def case_bar_necking(precision=_abi.PREC_FP64):
    """Round bar of the necking workload on a coarse mesh (4 x 4 O-grid, 20
    layers), pulled by its ramped end speed."""
    return meshes.bar_necking(n_core=4, n_ring=4, n_axial=20, precision=precision)


def case_plane_small(precision=_abi.PREC_FP64):
    """Plane-strain block (ElQua4N2D) with a distorted mesh and a random
    initial speed field."""
    return meshes.quad_block(4, 6, size=(1.2, 1.8), speed=60000.0, seed=13, distort=0.12, t_end=5e-6,
                             precision=precision, ts_freq=3)


def with_spare_material(desc):
    """The same model with a second, unused copy of its material.  An engine
    with one material reads it from the kernel parameters, one with several
    from global memory as a batch does; the two kernel families round the
    same arithmetic differently in the last bits, so a run that a batch must
    reproduce bit for bit is made on the several-materials family."""
    return desc.copy(materials=list(desc.materials) + [dict(desc.materials[0])])
