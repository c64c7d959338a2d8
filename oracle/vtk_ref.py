"""Restatement of the reference's VTK result files (test infrastructure only:
the checker of the engine's dnl_engine_write_vtk and the writer of the CPU
stand-in engine of the dnlPython tests; the engine never imports it).

Follows:
* the nodal extraction of point-state fields, Node::fieldScalar /
  fieldSymTensor2 with the _getFromIntegrationPoint macros (Node.C:244-365):
  at node n, sum over its elements (in element order) and their Gauss points
  of integrationPointsToNode(loc, g) * value, divided by the number of
  elements; the von Mises stress by dnlVonMises (Macros.h:71);
* the extrapolation weights of ElementData (ElHex8N3D.C:40-90,
  ElQua4NAx.C:37-58), written here in closed form: the shape function of
  Gauss point g's corner of the sub-element whose corners are the Gauss
  points, at node loc;
* the file layout of VtkInterface::headerWrite / nodesWrite / elementsWrite /
  dataWrite (VtkInterface.C:68-204), numbers as std::ostream prints a double
  by default (%g).

`parse(text)` reads a file back into its sections for numerical comparison.
"""
import math

import numpy as np

# the reference's VTK labels (Field.C:17-48) of the written fields:
# kind (0 scalar, 1 vector, 2 tensor) and source
FIELDS = {
    "coords": (1, "node", "coords"), "disp": (1, "node", "disp"), "dispInc": (1, "node", "u"),
    "speed": (1, "node", "speed"), "speedInc": (1, "node", "accel"),
    "density": (0, "ip", 27), "gamma": (0, "ip", 20), "gammaCumulate": (0, "ip", 21),
    "internalEnergy": (0, "ip", 25), "plasticStrain": (0, "ip", 18), "plasticStrainRate": (0, "ip", 19),
    "pressure": (0, "ip", 24), "T": (0, "ip", 23), "vonMises": (0, "ip", "vm"), "yield": (0, "ip", 22),
    "mass": (0, "node", "mass"), "PlasticStrain": (2, "ip", 12), "Strain": (2, "ip", 6), "Stress": (2, "ip", 0),
}

# the field list of the reference's settings file (Sources/dnlSettings/configuration.dnl,
# VtkFields) that Field::getField recognises (VtkInterface::initFields, VtkInterface.C:224-242)
DEFAULT_FIELDS = ["Stress", "Strain", "PlasticStrain", "vonMises", "yield", "pressure", "plasticStrain",
                  "plasticStrainRate", "gamma", "gammaCumulate", "speed"]


def _sign(n, k):
    # local coordinate sign of node / Gauss point n along axis k
    if k == 0:
        return 1 if (n & 3) in (1, 2) else -1
    if k == 1:
        return 1 if (n & 3) >= 2 else -1
    return 1 if n >= 4 else -1


def extrapolation_weights(npe):
    """[loc, g]: weight of Gauss point g's value at local node loc."""
    dim = 3 if npe == 8 else 2
    r3 = math.sqrt(3.0)
    w = np.zeros((npe, npe))
    for n in range(npe):
        for g in range(npe):
            m = sum(_sign(n, k) == _sign(g, k) for k in range(dim))
            if npe == 8:
                w[n, g] = [(5.0 - 3.0 * r3) / 4, (-1.0 + r3) / 4, (-1.0 - r3) / 4, (5.0 + 3.0 * r3) / 4][m]
            else:
                w[n, g] = [1.0 - r3 / 2, -0.5, 1.0 + r3 / 2][m]
    return w


def von_mises(ips):
    s1, s2, s3, s4, s5, s6 = ips[0], ips[3], ips[5], ips[1], ips[2], ips[4]
    return np.sqrt(((s1 - s2) ** 2 + (s1 - s3) ** 2 + (s2 - s3) ** 2 + 6.0 * (s4 * s4 + s5 * s5 + s6 * s6)) / 2)


def node_averages(conn, n_nodes, values):
    """values [k, n_ips] at the Gauss points (element-major) -> [k, n_nodes]."""
    conn = np.asarray(conn)
    nE, npe = conn.shape
    w = extrapolation_weights(npe)
    v = np.asarray(values, dtype=np.float64).reshape(-1, nE, npe)
    # contribution of element e to its local node loc: sum_g w[loc, g] v[e, g]
    contrib = np.einsum("lg,keg->kel", w, v)
    out = np.zeros((v.shape[0], n_nodes))
    count = np.bincount(conn.ravel(), minlength=n_nodes).astype(np.float64)
    # (summed local node by local node: the order of the element terms of a
    # node differs from the reference's only at the rounding level)
    for loc in range(npe):
        for k in range(v.shape[0]):
            np.add.at(out[k], conn[:, loc], contrib[k, :, loc])
    with np.errstate(invalid="ignore", divide="ignore"):
        return out / count


def _g(x):
    return "%g" % x


def write(path, time, coords, conn, vtk_type, node_fields, ips, fields, title="DynELA FEM Code v.4.0"):
    """node_fields: dict of 'disp', 'u', 'speed', 'accel', 'mass' ([n, 3])
    as the file must show them; ips [29, n_ips]."""
    conn = np.asarray(conn)
    nN, (nE, npe) = coords.shape[0], conn.shape
    lines = ["# vtk DataFile Version 4.0", title, "ASCII", "DATASET UNSTRUCTURED_GRID", "FIELD FieldData 1",
             "TIME 1 1 double", _g(time), f"POINTS {nN} float"]
    lines += [" ".join(_g(x) for x in row) for row in coords]
    lines += ["", f"CELLS {nE} {nE * (npe + 1)}"]
    lines += [f"{npe} " + "".join(f"{int(c)} " for c in row) for row in conn]
    lines += ["", f"CELL_TYPES {nE}"] + [str(vtk_type)] * nE + ["", f"POINT_DATA {nN}"]
    for name in fields:
        kind, src, what = FIELDS[name]
        if kind == 1:
            lines.append(f"VECTORS {name} float")
            v = coords if what == "coords" else node_fields[what]
            lines += [" ".join(_g(x) for x in row) for row in v]
        elif kind == 0:
            lines += [f"SCALARS {name} float", "LOOKUP_TABLE default"]
            if src == "node":
                vals = node_fields[what][:, 0]
            else:
                vals = node_averages(conn, nN, von_mises(ips)[None] if what == "vm" else ips[what][None])[0]
            lines += [_g(x) for x in vals]
        else:
            lines.append(f"TENSORS {name} float")
            t = node_averages(conn, nN, ips[what:what + 6])
            full = [0, 1, 2, 1, 3, 4, 2, 4, 5]
            lines += [" ".join(_g(t[c, i]) for c in full) for i in range(nN)]
    text = "\n".join(lines) + "\n\n"
    with open(path, "w") as f:
        f.write(text)
    return text


def parse(text):
    """Sections of a VTK file: header lines, time, points, cells, cell types
    and each point-data field (name -> array)."""
    lines = text.split("\n")
    out = {"header": lines[:6], "time": float(lines[6])}
    i = 7
    nN = int(lines[i].split()[1])
    out["points"] = np.array([[float(x) for x in lines[i + 1 + k].split()] for k in range(nN)])
    i += nN + 2
    assert lines[i].startswith("CELLS"), lines[i]
    nE = int(lines[i].split()[1])
    out["cells"] = np.array([[int(x) for x in lines[i + 1 + k].split()] for k in range(nE)])
    i += nE + 2
    assert lines[i].startswith("CELL_TYPES")
    out["cell_types"] = np.array([int(lines[i + 1 + k]) for k in range(nE)])
    i += nE + 2
    assert lines[i] == f"POINT_DATA {nN}", lines[i]
    i += 1
    fields = {}
    order = []
    while i < len(lines) and lines[i]:
        kind, name = lines[i].split()[:2]
        order.append(name)
        if kind == "SCALARS":
            fields[name] = np.array([float(lines[i + 2 + k]) for k in range(nN)])
            i += nN + 2
        else:
            fields[name] = np.array([[float(x) for x in lines[i + 1 + k].split()] for k in range(nN)])
            i += nN + 1
    out["fields"], out["order"] = fields, order
    return out


def compare(a, b, rtol=2e-5):
    """Largest difference between two parsed files, relative to each field's
    largest magnitude (the files hold 6 significant digits); the structure
    (cells, cell types, field order) must be equal."""
    assert np.array_equal(a["cells"], b["cells"]) and np.array_equal(a["cell_types"], b["cell_types"])
    assert a["order"] == b["order"], (a["order"], b["order"])
    worst = {"time": abs(a["time"] - b["time"]) / max(abs(b["time"]), 1e-300),
             "points": np.abs(a["points"] - b["points"]).max() / max(np.abs(b["points"]).max(), 1e-300)}
    for k in b["fields"]:
        x, y = a["fields"][k], b["fields"][k]
        worst[k] = float(np.abs(x - y).max() / max(np.abs(y).max(), 1e-30))
    return worst
