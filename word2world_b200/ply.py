"""PLY files of Gaussian parameters, in the reference's layout
(``GaussianIO.save_as_ply``, ``GaussianIO.py:9-46``): the on-disk format of
the scenes a serving loop loads.

One ``vertex`` element, every property ``float`` (4-byte), binary
little-endian, in this order:

* ``x y z`` -- the mean;
* ``sh_coefficients_dc_0..2`` -- the DC colour coefficients;
* ``sh_coefficients_ac_0..3K-1`` -- the K rest coefficients per channel,
  channel-major: property ``c*K + k`` holds coefficient k of channel c (the
  reference flattens ``sh.transpose(1, 2)``, ``misc_utils.py:41-43``);
* ``opacity`` -- the opacity logit;
* ``svec_0..2`` -- the log-scales;
* ``quaternion_0..3`` -- the rotation (w, x, y, z), unnormalised.

The reference writes through the third-party ``plyfile`` package (absent
here); this module writes the same bytes with numpy.  ``load_ply`` inverts
``save_ply`` exactly.  The reference's own loader (``GaussianIO.py:48-74``)
reads the rest coefficients coefficient-major (property ``k*3 + c``), the
transpose of what its writer wrote, and its caller passes it an extra
argument (``gaussians_handler.py:92``); neither is reproduced.
"""
from __future__ import annotations

import numpy as np

_TYPES = {"char": "i1", "int8": "i1", "uchar": "u1", "uint8": "u1", "short": "i2", "int16": "i2",
          "ushort": "u2", "uint16": "u2", "int": "i4", "int32": "i4", "uint": "u4", "uint32": "u4",
          "float": "f4", "float32": "f4", "double": "f8", "float64": "f8"}


def property_names(K: int) -> list:
    """Vertex property names in file order for K rest SH coefficients per channel."""
    names = ["x", "y", "z"] + [f"sh_coefficients_dc_{i}" for i in range(3)]
    names += [f"sh_coefficients_ac_{i}" for i in range(3 * K)]
    names += ["opacity"] + [f"svec_{i}" for i in range(3)] + [f"quaternion_{i}" for i in range(4)]
    return names


def _np(a):
    if hasattr(a, "detach"):
        a = a.detach().cpu().numpy()
    return np.asarray(a, dtype=np.float32)


def save_ply(path, mean, sh_dc, sh_ac, opacity, svec, quaternion):
    """Write P Gaussians: mean [P,3], sh_dc [P,1,3], sh_ac [P,K,3], opacity
    [P,1] logits, svec [P,3] log-scales, quaternion [P,4] (numpy arrays or
    tensors)."""
    import os
    mean, sh_dc, sh_ac = _np(mean), _np(sh_dc), _np(sh_ac)
    opacity, svec, quaternion = _np(opacity), _np(svec), _np(quaternion)
    P = mean.shape[0]
    sh_ac = sh_ac.reshape(P, -1, 3)
    K = sh_ac.shape[1]
    cols = [mean.reshape(P, 3), sh_dc.reshape(P, 1, 3).transpose(0, 2, 1).reshape(P, 3),
            sh_ac.transpose(0, 2, 1).reshape(P, 3 * K), opacity.reshape(P, 1), svec.reshape(P, 3),
            quaternion.reshape(P, 4)]
    data = np.ascontiguousarray(np.concatenate(cols, axis=1), dtype="<f4")
    names = property_names(K)
    header = ["ply", "format binary_little_endian 1.0", f"element vertex {P}"]
    header += [f"property float {n}" for n in names] + ["end_header"]
    d = os.path.dirname(os.path.abspath(path))
    os.makedirs(d, exist_ok=True)
    with open(path, "wb") as f:
        f.write(("\n".join(header) + "\n").encode("ascii"))
        f.write(data.tobytes())


def _read_header(f):
    line = f.readline().strip()
    if line != b"ply":
        raise ValueError("not a PLY file")
    fmt, elements, cur = None, [], None
    while True:
        raw = f.readline()
        if not raw:
            raise ValueError("PLY header ends before end_header")
        tok = raw.decode("ascii").split()
        if not tok or tok[0] in ("comment", "obj_info"):
            continue
        if tok[0] == "format":
            fmt = tok[1]
        elif tok[0] == "element":
            cur = {"name": tok[1], "count": int(tok[2]), "props": []}
            elements.append(cur)
        elif tok[0] == "property":
            if tok[1] == "list":
                raise ValueError("list properties are not supported")
            cur["props"].append((tok[2], _TYPES[tok[1]]))
        elif tok[0] == "end_header":
            return fmt, elements


def read_vertices(path) -> np.ndarray:
    """The vertex element as a numpy structured array (binary little- or
    big-endian, or ascii)."""
    with open(path, "rb") as f:
        fmt, elements = _read_header(f)
        out = None
        for el in elements:
            if fmt == "ascii":
                dt = np.dtype([(n, t) for n, t in el["props"]])
                vals = np.array([[float(x) for x in f.readline().split()] for _ in range(el["count"])],
                                dtype=np.float64).reshape(el["count"], len(el["props"]))
                arr = np.zeros(el["count"], dt)
                for j, (n, _) in enumerate(el["props"]):
                    arr[n] = vals[:, j]
            else:
                bo = "<" if fmt == "binary_little_endian" else ">"
                dt = np.dtype([(n, bo + t) for n, t in el["props"]])
                arr = np.frombuffer(f.read(dt.itemsize * el["count"]), dtype=dt, count=el["count"])
            if el["name"] == "vertex":
                out = arr
        if out is None:
            raise ValueError("no vertex element")
        return out


def load_ply(path) -> dict:
    """The arrays ``save_ply`` wrote: mean [P,3], sh_dc [P,1,3], sh_ac
    [P,K,3], opacity [P,1], svec [P,3], quaternion [P,4] (float32)."""
    v = read_vertices(path)
    names = v.dtype.names
    P = v.shape[0]
    col = lambda n: np.asarray(v[n], dtype=np.float32)
    K3 = sum(1 for n in names if n.startswith("sh_coefficients_ac_"))
    if K3 % 3:
        raise ValueError("rest SH coefficients must come in threes")
    K = K3 // 3
    ac = np.stack([col(f"sh_coefficients_ac_{i}") for i in range(3 * K)], axis=1) if K else np.zeros((P, 0))
    return {
        "mean": np.stack([col("x"), col("y"), col("z")], axis=1),
        "sh_dc": np.stack([col(f"sh_coefficients_dc_{i}") for i in range(3)], axis=1).reshape(P, 1, 3),
        "sh_ac": ac.reshape(P, 3, K).transpose(0, 2, 1).copy(),
        "opacity": col("opacity").reshape(P, 1),
        "svec": np.stack([col(f"svec_{i}") for i in range(3)], axis=1),
        "quaternion": np.stack([col(f"quaternion_{i}") for i in range(4)], axis=1),
    }
