"""PLY IO in the reference's layout (GaussianIO.py:9-46): header, property
order, channel-major rest coefficients, exact round trip."""
import os

import numpy as np

from word2world_b200 import ply, scenes


def test_round_trip_and_layout(tmp_path):
    sc = scenes.make_scene(257, seed=9)
    path = os.path.join(tmp_path, "sub", "scene.ply")
    ply.save_ply(path, sc.mean, sc.sh_dc, sc.sh_ac, sc.opacity, sc.svec, sc.quaternion)
    raw = open(path, "rb").read()
    head, body = raw.split(b"end_header\n", 1)
    lines = head.decode().splitlines()
    assert lines[:3] == ["ply", "format binary_little_endian 1.0", "element vertex 257"]
    names = [l.split()[2] for l in lines[3:]]
    assert all(l.split()[1] == "float" for l in lines[3:])
    assert names == ply.property_names(15) and len(names) == 59
    assert names[:6] == ["x", "y", "z", "sh_coefficients_dc_0", "sh_coefficients_dc_1", "sh_coefficients_dc_2"]
    assert names[-8:] == ["opacity", "svec_0", "svec_1", "svec_2", "quaternion_0", "quaternion_1", "quaternion_2",
                          "quaternion_3"]
    assert len(body) == 257 * 59 * 4
    rows = np.frombuffer(body, dtype="<f4").reshape(257, 59)
    # channel-major rest coefficients: property c*15 + k is coefficient k of channel c
    ac = np.asarray(sc.sh_ac, np.float32)
    assert rows[5, 6 + 2 * 15 + 7] == ac[5, 7, 2]
    assert rows[5, 6 + 1] == np.float32(ac[5, 1, 0])
    d = ply.load_ply(path)
    for k, want in (("mean", sc.mean), ("sh_dc", sc.sh_dc), ("sh_ac", sc.sh_ac), ("opacity", sc.opacity),
                    ("svec", sc.svec), ("quaternion", sc.quaternion)):
        assert d[k].shape == np.shape(want) and d[k].dtype == np.float32
        assert np.array_equal(d[k], np.asarray(want, np.float32)), k


def test_ascii_and_degree0(tmp_path):
    P = 3
    path = os.path.join(tmp_path, "a.ply")
    names = ply.property_names(0)
    with open(path, "w") as f:
        f.write("ply\nformat ascii 1.0\ncomment written by hand\nelement vertex 3\n")
        f.write("".join(f"property float {n}\n" for n in names) + "end_header\n")
        for i in range(P):
            f.write(" ".join(str(float(i * 100 + j)) for j in range(len(names))) + "\n")
    d = ply.load_ply(path)
    assert d["sh_ac"].shape == (3, 0, 3)
    assert d["mean"][2].tolist() == [200.0, 201.0, 202.0]
    assert d["quaternion"][1].tolist() == [110.0, 111.0, 112.0, 113.0]
