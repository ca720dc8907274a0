"""ORACLE — test infrastructure only.

CPU restatement of the reference's indexed OBJ parse,
OBJReader._parse_indexed (scene/io/obj_reader.py:345-441), used as the
checker of the device parser (rx_obj_* in libroxy_cuda.so) and as the CPU
baseline of the OBJ workload in bench.py.  Only the tests, smoke() and
bench.py's CPU-baseline leg use it.

It reads the text the way the reference does: universal-newline lines
(obj_reader.py:384 `for line in f` on a text-mode file), str.split() tokens,
float() / int() conversions, 1-based and relative indices (`_idx`,
obj_reader.py:354-356), fan triangulation (obj_reader.py:411-417) and group
ids in order of first usemtl (obj_reader.py:358-362, 400-403).

Parity pin: tests/test_oracle_golden.py checks it against
tests/golden/obj_*.npz, which tests/golden/make_golden.py produced by running
the reference's OBJReader on the same text.
"""
import io

import numpy as np


def _index(raw, count):
    i = int(raw)
    return i - 1 if i > 0 else count + i


def parse_indexed(text):
    """text (str or bytes) -> dict of the IndexedMesh arrays, the group names,
    the groups that received triangles and the unrecognised tokens."""
    if isinstance(text, (bytes, bytearray)):
        text = text.decode("utf-8")
    pos, nrm, uv = [], [], []
    tp, tn, tu, tg = [], [], [], []
    groups, gid_of = ["default"], {"default": 0}
    used, unknown = set(), []
    mtl, gid = "default", 0
    for line in io.StringIO(text, newline=None):
        parts = line.split()
        if not parts or parts[0].startswith("#"):
            continue
        key = parts[0]
        if key == "v":
            pos.append((float(parts[1]), float(parts[2]), float(parts[3])))
        elif key == "vn":
            nrm.append((float(parts[1]), float(parts[2]), float(parts[3])))
        elif key == "vt":
            uv.append((float(parts[1]), float(parts[2])))
        elif key == "usemtl":
            mtl = parts[1] if len(parts) > 1 else "default"
            if mtl not in gid_of:
                gid_of[mtl] = len(groups)
                groups.append(mtl)
            gid = gid_of[mtl]
        elif key == "f":
            corners = []
            for tok in parts[1:]:
                f = tok.split("/")
                corners.append((_index(f[0], len(pos)),
                                _index(f[1], len(uv)) if len(f) > 1 and f[1] else -1,
                                _index(f[2], len(nrm)) if len(f) > 2 and f[2] else -1))
            for k in range(1, len(corners) - 1):
                a, b, c = corners[0], corners[k], corners[k + 1]
                tp.append((a[0], b[0], c[0]))
                tu.append((a[1], b[1], c[1]))
                tn.append((a[2], b[2], c[2]))
                tg.append(gid)
                used.add(mtl)
        elif key in ("mtllib", "o", "g", "s"):
            continue
        else:
            unknown.append(key)
    return {
        "positions": np.asarray(pos, np.float64).reshape(-1, 3),
        "normals": np.asarray(nrm, np.float64).reshape(-1, 3),
        "uvs": np.asarray(uv, np.float64).reshape(-1, 2),
        "tri_pos_idx": np.asarray(tp, np.int32).reshape(-1, 3),
        "tri_normal_idx": np.asarray(tn, np.int32).reshape(-1, 3),
        "tri_uv_idx": np.asarray(tu, np.int32).reshape(-1, 3),
        "tri_group_idx": np.asarray(tg, np.int32).reshape(-1),
        "groups": groups,
        "used_groups": used,
        "unknown": unknown,
    }
