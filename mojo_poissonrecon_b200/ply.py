"""PLY output of reconstructed meshes (and a reader for the files it writes).

The reference returns meshes as arrays only (its README points users to their
own writers); upstream PoissonRecon writes PLY with float coordinates and, on
request, each vertex's sample density as a `value` property.  `write_ply`
writes a `Mesh` (NumPy arrays, or CUDA tensors from `device_out=True`) the same
way: binary little-endian by default (ASCII on request), coordinates as
`float` (or `double`), the density as `value` when asked for, faces as
`list uchar int vertex_indices`, and the iso-value in a comment.  `read_ply`
reads ASCII and binary little-endian files with scalar vertex properties and
one list property per face, enough to round-trip these files and to load the
common ones.
"""

from __future__ import annotations

import os

import numpy as np

_SCALARS = {
    "char": "i1", "int8": "i1", "uchar": "u1", "uint8": "u1",
    "short": "i2", "int16": "i2", "ushort": "u2", "uint16": "u2",
    "int": "i4", "int32": "i4", "uint": "u4", "uint32": "u4",
    "float": "f4", "float32": "f4", "double": "f8", "float64": "f8",
}


def _numpy(a) -> np.ndarray:
    if hasattr(a, "detach"):  # torch tensor, on the host or a device
        return a.detach().cpu().numpy()
    return np.asarray(a)


_PLY_TYPES = {np.dtype("u1"): "uchar", np.dtype("i1"): "char", np.dtype("u2"): "ushort", np.dtype("i2"): "short",
              np.dtype("u4"): "uint", np.dtype("i4"): "int", np.dtype("f4"): "float", np.dtype("f8"): "double"}


def write_ply(path, mesh, *, binary: bool = True, coordinates: str = "float", density: bool = True,
              properties: dict | None = None, comment: str | None = None) -> None:
    """Write `mesh` (vertices (V, 3), faces (F, 3), density (V,)) to `path`.

    coordinates: "float" or "double" for x, y, z (and the density `value`).
    density: write each vertex's density as a `value` property.
    properties: further per-vertex scalars {name: (V,) array}, written after
    them in the array's own type (uint8, int8, (u)int16, (u)int32, float32,
    float64; e.g. colours as uint8 "red", "green", "blue").
    Raises ValueError on malformed arrays or face indices outside [0, V)."""
    if coordinates not in ("float", "double"):
        raise ValueError("coordinates must be 'float' or 'double'")
    vertices = _numpy(mesh.vertices).astype(np.float64, copy=False).reshape(-1, 3)
    faces = _numpy(mesh.faces).reshape(-1, 3)
    values = _numpy(mesh.density).astype(np.float64, copy=False).reshape(-1) if density else None
    nv, nf = vertices.shape[0], faces.shape[0]
    if values is not None and values.shape[0] != nv:
        raise ValueError("density must have one value per vertex")
    if nf and (faces.min() < 0 or faces.max() >= nv):
        raise ValueError("face indices must lie in [0, vertex count)")
    extra = []
    for name, values_k in (properties or {}).items():
        arr = _numpy(values_k).reshape(-1)
        if arr.dtype not in _PLY_TYPES:
            raise ValueError(f"property {name!r}: unsupported type {arr.dtype}")
        if arr.shape[0] != nv:
            raise ValueError(f"property {name!r} must have one value per vertex")
        if name in ("x", "y", "z", "value") or not name.isidentifier():
            raise ValueError(f"property name {name!r} is reserved or not a plain identifier")
        extra.append((name, arr))
    ctype = "f4" if coordinates == "float" else "f8"

    header = ["ply", "format " + ("binary_little_endian" if binary else "ascii") + " 1.0",
              "comment written by mojo_poissonrecon_b200"]
    iso = getattr(mesh, "iso_value", None)
    if iso is not None:
        header.append(f"comment iso_value {float(iso)!r}")
    if comment:
        header.extend("comment " + line for line in str(comment).splitlines())
    header.append(f"element vertex {nv}")
    header.extend(f"property {coordinates} {axis}" for axis in "xyz")
    if values is not None:
        header.append(f"property {coordinates} value")
    header.extend(f"property {_PLY_TYPES[arr.dtype]} {name}" for name, arr in extra)
    header.append(f"element face {nf}")
    header.append("property list uchar int vertex_indices")
    header.append("end_header")
    head = ("\n".join(header) + "\n").encode("ascii")

    fields = [("x", "<" + ctype), ("y", "<" + ctype), ("z", "<" + ctype)]
    if values is not None:
        fields.append(("value", "<" + ctype))
    fields.extend((name, arr.dtype.newbyteorder("<")) for name, arr in extra)
    vrec = np.empty(nv, dtype=fields)
    vrec["x"], vrec["y"], vrec["z"] = vertices[:, 0], vertices[:, 1], vertices[:, 2]
    if values is not None:
        vrec["value"] = values
    for name, arr in extra:
        vrec[name] = arr
    frec = np.empty(nf, dtype=[("n", "u1"), ("v", "<i4", (3,))])
    frec["n"] = 3
    frec["v"] = faces

    tmp = os.fspath(path)
    with open(tmp, "wb") as f:
        f.write(head)
        if binary:
            f.write(vrec.tobytes())
            f.write(frec.tobytes())
        else:  # shortest round-tripping decimal of each stored value, integers as integers
            cfmt = "%.9g" if coordinates == "float" else "%.17g"
            fmts = [cfmt] * (3 + (values is not None))
            fmts += ["%d" if arr.dtype.kind in "iu" else ("%.9g" if arr.dtype == np.float32 else "%.17g")
                     for _, arr in extra]
            if nv:
                rows = zip(*([vrec[name] for name, _ in fields]))
                f.write("".join(" ".join(fm % v for fm, v in zip(fmts, row)) + "\n" for row in rows).encode("ascii"))
            if nf:
                np.savetxt(f, np.column_stack([np.full(nf, 3), faces]), fmt="%d")


def read_ply(path) -> dict:
    """Read a PLY file: {"vertices": (V, 3) float64, "faces": (F, k) int64 (k the
    common polygon size; ValueError when sizes differ), "properties": {name:
    (V,) array} for the vertex's other scalar properties, "comments": [...]}."""
    with open(os.fspath(path), "rb") as f:
        data = f.read()
    end = data.find(b"end_header")
    if not data.startswith(b"ply") or end < 0:
        raise ValueError("not a PLY file")
    body_start = data.index(b"\n", end) + 1
    lines = data[:end].decode("ascii").splitlines()
    fmt, comments, elements = None, [], []
    for line in lines[1:]:
        words = line.split()
        if not words:
            continue
        if words[0] == "format":
            fmt = words[1]
        elif words[0] == "comment":
            comments.append(line[len("comment "):])
        elif words[0] == "element":
            elements.append({"name": words[1], "count": int(words[2]), "props": []})
        elif words[0] == "property":
            if words[1] == "list":
                elements[-1]["props"].append((words[4], ("list", _SCALARS[words[2]], _SCALARS[words[3]])))
            else:
                elements[-1]["props"].append((words[2], _SCALARS[words[1]]))
    if fmt not in ("ascii", "binary_little_endian"):
        raise ValueError(f"unsupported PLY format {fmt!r}")
    out = {"vertices": np.empty((0, 3)), "faces": np.empty((0, 3), np.int64), "properties": {},
           "comments": comments}
    if fmt == "ascii":
        tokens = data[body_start:].split()
        pos = 0
        for el in elements:
            rows = []
            for _ in range(el["count"]):
                row = {}
                for name, kind in el["props"]:
                    if isinstance(kind, tuple):
                        k = int(tokens[pos])
                        row[name] = np.array(tokens[pos + 1:pos + 1 + k], dtype=np.int64)
                        pos += 1 + k
                    else:
                        row[name] = float(tokens[pos])
                        pos += 1
                rows.append(row)
            if all(not isinstance(kind, tuple) for _, kind in el["props"]):  # values of the declared types
                dt = np.dtype([(name, kind) for name, kind in el["props"]])
                rows = np.array([tuple(r[name] for name, _ in el["props"]) for r in rows], dtype=dt)
            _store(out, el, rows)
        return out
    pos = body_start
    for el in elements:
        if all(not isinstance(kind, tuple) for _, kind in el["props"]):
            dt = np.dtype([(name, "<" + kind) for name, kind in el["props"]])
            rec = np.frombuffer(data, dtype=dt, count=el["count"], offset=pos)
            pos += dt.itemsize * el["count"]
            _store(out, el, rec)
        else:  # one list property (faces): fixed-size rows when every polygon has the same size
            (name, (_, count_t, index_t)), = [(n, k) for n, k in el["props"] if isinstance(k, tuple)]
            if len(el["props"]) != 1:
                raise ValueError("faces with properties besides the index list are not supported")
            rows = []
            csize, isize = np.dtype(count_t).itemsize, np.dtype(index_t).itemsize
            for _ in range(el["count"]):
                k = int(np.frombuffer(data, dtype="<" + count_t, count=1, offset=pos)[0])
                rows.append({name: np.frombuffer(data, dtype="<" + index_t, count=k, offset=pos + csize)
                             .astype(np.int64)})
                pos += csize + k * isize
            _store(out, el, rows)
    return out


def _store(out: dict, el: dict, rows) -> None:
    if el["name"] == "vertex":
        names = [name for name, _ in el["props"]]
        col = (lambda n: rows[n]) if isinstance(rows, np.ndarray) else \
            (lambda n: np.array([r[n] for r in rows], dtype=np.float64))
        if el["count"]:
            out["vertices"] = np.column_stack([col(a) for a in "xyz"]).astype(np.float64)
        out["properties"] = {n: np.asarray(col(n)) for n in names if n not in ("x", "y", "z")}
    elif el["name"] == "face":
        lists = [r[el["props"][0][0]] for r in rows]
        if lists:
            sizes = {len(v) for v in lists}
            if len(sizes) != 1:
                raise ValueError("faces of different sizes")
            out["faces"] = np.stack(lists).astype(np.int64)
