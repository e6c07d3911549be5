"""PLY blobs for the ingest tests: well-formed files of every SH degree and the
header edge cases of the reference loader (src/GS_ply.ts:58-132), plus the
tie rule used to compare two activations of the same file.

Every blob is built here from seeded random columns; nothing is read from
disk.  A case is (name, blob, accepted) where `accepted` says whether the
reference loader packs the file (True) or throws / would pack NaN (False).
"""
from __future__ import annotations

import numpy as np

BASE = ["x", "y", "z", "nx", "ny", "nz"]


def _names(degree: int):
    per = (degree + 1) ** 2 - 1
    return (BASE + ["f_dc_0", "f_dc_1", "f_dc_2"] + [f"f_rest_{i}" for i in range(3 * per)]
            + ["opacity", "scale_0", "scale_1", "scale_2", "rot_0", "rot_1", "rot_2", "rot_3"])


def _values(name: str, n: int, rng) -> np.ndarray:
    if name.startswith("scale_"):
        return rng.uniform(-6.0, -1.0, n)
    if name == "opacity":
        return rng.normal(0.0, 2.0, n)
    if name.startswith("rot_"):
        return rng.normal(0.0, 1.0, n)
    if name.startswith("f_"):
        return rng.normal(0.0, 0.4, n)
    return rng.normal(0.0, 1.5, n)


def build(props, n: int, seed: int = 1, header_extra=(), body_props=None, newline="\n",
          vertex_lines=None, trailing: int = 64) -> bytes:
    """props: [(type, name)] declared in order.  body_props: [(type, name)]
    actually stored per vertex (defaults to the float/uchar ones of props, in
    declared order); a uchar column stores round(255 * u), u in [0, 1)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    if body_props is None:
        body_props = [(t, nm) for t, nm in props if t in ("float", "uchar")]
    lines = ["ply", "format binary_little_endian 1.0"]
    lines += list(vertex_lines) if vertex_lines is not None else [f"element vertex {n}"]
    lines += list(header_extra)
    lines += [f"property {t} {nm}" for t, nm in props]
    lines += ["end_header"]
    head = (newline.join(lines) + "\n").encode("ascii")
    cols = []
    for t, nm in body_props:
        if t == "float":
            cols.append(("<f4", _values(nm, n, rng).astype("<f4")))
        else:
            cols.append(("u1", rng.integers(0, 256, n).astype("u1")))
    dt = np.dtype([(f"c{i}", c[0]) for i, c in enumerate(cols)])
    body = np.zeros(n, dtype=dt)
    for i, c in enumerate(cols):
        body[f"c{i}"] = c[1]
    # trailing bytes keep the 50-byte header chunk inside the file for tiny n
    return head + body.tobytes() + b"\0" * trailing


def standard(n: int, degree: int = 3, seed: int = 1) -> bytes:
    return build([("float", nm) for nm in _names(degree)], n, seed)


def cases():
    """(name, blob, accepted) for the header rules and edge cases."""
    std3 = [("float", nm) for nm in _names(3)]
    out = []
    for d in range(4):
        out.append((f"degree{d}", standard(37, d, seed=10 + d), True))
    out.append(("zero_vertices", standard(0, 3), True))
    # a uchar property in front: every float after it is unaligned
    out.append(("uchar_first", build([("uchar", "red")] + std3, 29, seed=3), True))
    # uchar-typed SH and opacity columns (read as byte / 255)
    mixed = [(("uchar" if nm in ("f_dc_1", "opacity", "f_rest_7") else "float"), nm) for nm in _names(3)]
    out.append(("uchar_values", build(mixed, 23, seed=4), True))
    # shuffled declaration order
    rng = np.random.Generator(np.random.PCG64(5))
    sh = list(std3)
    rng.shuffle(sh)
    out.append(("shuffled", build(sh, 31, seed=5), True))
    # a repeated name keeps its first place and takes the later type
    dup = std3[:3] + [("uchar", "scale_0")] + std3[3:]
    body = [(t, nm) for t, nm in std3[:3]] + [("float", "scale_0")] + \
        [(t, nm) for t, nm in std3[3:] if nm != "scale_0"]
    out.append(("duplicate_name", build(dup, 17, seed=6, body_props=body), True))
    # array-index names come first in ascending order
    idx = std3[:2] + [("float", "7")] + std3[2:5] + [("float", "0")] + std3[5:]
    body = [("float", "0"), ("float", "7")] + std3
    out.append(("index_names", build(idx, 19, seed=7, body_props=body), True))
    # "__proto__" creates no property (and no bytes)
    out.append(("proto_name", build(std3[:4] + [("float", "__proto__")] + std3[4:], 13, seed=8, body_props=std3),
                True))
    # other types are not read and take no bytes; a face list is harmless
    out.append(("double_and_list", build(std3 + [("double", "extra")], 21, seed=9, body_props=std3,
                                         header_extra=[]), True))
    out.append(("face_element", build(std3, 11, seed=12, body_props=std3) .replace(
        b"end_header\n", b"element face 0\nproperty list uchar int vertex_indices\nend_header\n", 1), True))
    # CRLF line endings, comments, two vertex-count lines (the last wins)
    out.append(("crlf", build(std3, 15, seed=13, newline="\r\n"), True))
    out.append(("comments", build(std3, 9, seed=14, header_extra=["comment made by a test", "obj_info x"]), True))
    out.append(("two_counts", build(std3, 12, seed=15, vertex_lines=["element vertex 5", "element vertex 12"]), True))
    # errors
    out.append(("no_end_header", standard(5).replace(b"end_header", b"end_headex"), False))
    full = standard(1, 3, seed=16)
    head_len = full.index(b"end_header") + 11
    out.append(("chunk_past_eof", full[:head_len], False))
    out.append(("non_ascii", non_ascii_blob(), False))
    out.append(("missing_opacity", build([p for p in std3 if p[1] != "opacity"], 8, seed=18), False))
    out.append(("bad_degree", build(std3[:15] + std3[-8:], 8, seed=19), False))
    out.append(("short_body", standard(40, 3, seed=20)[:-64 - 300], False))
    out.append(("double_position", build([("double", "x")] + std3[1:], 8, seed=21,
                                         body_props=std3[1:]), False))
    return out


def non_ascii_blob() -> bytes:
    std3 = [("float", nm) for nm in _names(3)]
    b = build(std3, 4, seed=17, header_extra=["comment cafe"])
    return b.replace(b"comment cafe", b"comment caf\xc3\xa9")


def exact_words(pg) -> np.ndarray:
    """The double-precision values behind each packed word of a
    PackedGaussians mirror (NaN for padding words)."""
    d = pg.gaussianData
    n = pg.numGaussians
    words = pg.gaussiansBuffer.shape[1] if n else 0
    ex = np.full((n, words), np.nan)
    if n == 0:
        return ex
    ex[:, 0:3] = d["position"]
    ex[:, 4:7] = d["scale"]
    ex[:, 8:12] = d["rotQuat"]
    ex[:, 12] = d["opacity"]
    sh = d["shCoeffs"]
    for j in range(sh.shape[1]):
        ex[:, 16 + 4 * j:19 + 4 * j] = sh[:, j, :]
    return ex


def check_activation(got: np.ndarray, want: np.ndarray, exact64: np.ndarray | None = None, ulps64: int = 4):
    """Asserts two packings of one file are equal bit for bit, except words
    whose double-precision value (exact64, same shape, NaN where not
    applicable) lies within `ulps64` double ulps of a binary32 rounding
    boundary: there two correct `exp` implementations may round apart."""
    g = got.view(np.uint32)
    w = want.view(np.uint32)
    bad = np.argwhere(g != w)
    if bad.size == 0:
        return 0
    assert exact64 is not None, f"{len(bad)} words differ, first at {bad[0].tolist()}"
    for r, c in bad:
        v = float(exact64[r, c])
        a, b = sorted((float(got[r, c]), float(want[r, c])))
        assert np.nextafter(np.float32(a), np.float32(np.inf)) == np.float32(b), (r, c, a, b)
        mid = (a + b) / 2.0
        assert abs(v - mid) <= ulps64 * np.spacing(abs(mid)), (r, c, v, a, b)
    return len(bad)
