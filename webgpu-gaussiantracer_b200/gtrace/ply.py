"""3DGS PLY ingest and packing: host-side mirror of the reference's loader.

Mirrors ``PackedGaussians`` (src/GS_ply.ts:39-253) and the std430 packing
rules it uses (src/GS_packing.ts:146-174, 233-245), vectorised with numpy:

* header: ``element vertex N`` and ``property <type> <name>`` lines; vertex
  data starts one byte after ``end_header`` (src/GS_ply.ts:58-111);
* properties are read in header order, ``float`` as little-endian f32 and
  ``uchar`` as byte / 255 (:113-132);
* activation in double precision (:225-235): ``scale = exp(raw)``, the
  quaternion divided by its norm, ``opacity = 1 / (1 + exp(-raw))``;
* SH order (:188-196): ``sh[0] = f_dc_0..2`` and
  ``sh[i+1] = (f_rest_i, f_rest_{n+i}, f_rest_{2n+i})`` with n = #f_rest / 3;
* packed record (:199-207): position vec3 @0, scale vec3 @16,
  rotation vec4 @32, opacity f32 @48, sh vec3[n_sh] @64 with array stride 16;
  320 bytes for SH degree 3.

``write_ply`` writes the same format (pre-activation values), so scenes made
here load in the reference's own TypeScript host unchanged.
"""
from __future__ import annotations

import math
import re
from dataclasses import dataclass, field

import numpy as np

_PLY_TYPES = {"float": "<f4", "uchar": "u1", "double": "<f8", "int": "<i4",
              "uint": "<u4", "short": "<i2", "ushort": "<u2", "char": "i1"}


class PlyError(ValueError):
    """Raised for a file the reference's loader could not read either."""


_JS_SPACE = " \t\n\v\f\r"
_PROPERTY_RE = re.compile(r"([A-Za-z0-9_]+)[ \t\n\v\f\r]+([A-Za-z0-9_]+)[ \t\n\v\f\r]+([A-Za-z0-9_]+)")


def _array_index(name: str):
    """The value of a canonical array-index key ("0", or digits without a
    leading zero below 2^32 - 1), else None: such keys of a JS object come
    first, in ascending order."""
    if not name or not name.isascii() or not name.isdigit() or (len(name) > 1 and name[0] == "0"):
        return None
    v = int(name)
    return v if v < 4294967295 else None


def _decode_header(buf: bytes):
    """Returns (vertex_count, [(name, type)], data_offset) (src/GS_ply.ts:58-111).

    The reference reads the header in 50-byte chunks until the text holds
    ``end_header`` (a file that ends inside that chunk makes its 50-byte view
    throw), scans the trimmed lines of those chunks up to a line equal to
    ``end_header``, and keeps ``propertyTypes`` as a JS object: array-index
    names first in ascending order, then the others in first-insertion order,
    a repeated name keeping its place with the later type, ``__proto__``
    creating no entry.  The body starts one byte past the first
    ``end_header``.  The header must be ASCII here (the reference takes byte
    offsets from UTF-8-decoded text, which only agree for ASCII)."""
    pos = buf.find(b"end_header")
    if pos < 0:
        raise PlyError("PLY header has no end_header")
    chunk_end = (pos + 10 + 49) // 50 * 50
    if chunk_end > len(buf):
        raise PlyError("the file ends inside the 50-byte header chunk that holds end_header")
    if any(b >= 0x80 for b in buf[:pos]):
        raise PlyError("the PLY header is not ASCII")
    text = buf[:chunk_end].decode("latin-1")
    count = 0
    named: dict[str, str] = {}
    indexed: dict[int, tuple[str, str]] = {}
    for raw in text.split("\n"):
        line = raw.strip(_JS_SPACE)
        if line.startswith("element vertex"):
            m = re.search(r"[0-9]+", line)
            if m:
                count = int(m.group(0))
        elif line.startswith("property"):
            m = _PROPERTY_RE.search(line)
            if m and m.group(3) != "__proto__":
                name, typ = m.group(3), m.group(2)
                idx = _array_index(name)
                if idx is not None:
                    indexed[idx] = (name, typ)
                else:
                    named[name] = typ  # a dict keeps the first insertion's place
        elif line == "end_header":
            break
    props = [indexed[i] for i in sorted(indexed)] + list(named.items())
    return count, props, pos + 10 + 1


def _sh_feature_order(n_rest: int) -> list[str]:
    per_color = n_rest // 3
    order = [f"f_dc_{c}" for c in range(3)]
    for i in range(per_color):
        for c in range(3):
            order.append(f"f_rest_{c * per_color + i}")
    return order


def record_stride(sh_degree: int) -> int:
    """Packed record size in bytes for an SH degree (std430 rules)."""
    n_sh = (sh_degree + 1) ** 2
    return 64 + 16 * n_sh


@dataclass
class PackedGaussians:
    """Reads a 3DGS PLY blob and packs it the way the shaders expect.

    Attributes mirror the reference class: ``numGaussians``,
    ``sphericalHarmonicsDegree``, ``gaussiansBuffer`` (packed records, float32
    array of shape (n, stride/4)), ``positionsBuffer`` (n x 4 float32, vec3 at
    stride 16) and ``gaussianData`` (activated values as float64 arrays:
    position, scale, rotQuat, opacity, shCoeffs).
    """

    array_buffer: bytes
    numGaussians: int = field(init=False)
    sphericalHarmonicsDegree: int = field(init=False)
    gaussiansBuffer: np.ndarray = field(init=False, repr=False)
    positionsBuffer: np.ndarray = field(init=False, repr=False)
    gaussianData: dict = field(init=False, repr=False)

    def __post_init__(self):
        buf = bytes(self.array_buffer) if not isinstance(self.array_buffer, bytes) else self.array_buffer
        count, props, offset = _decode_header(buf)
        n_rest = sum(1 for name, _ in props if name.startswith("f_rest_"))
        per_color = n_rest / 3
        degree = math.sqrt(per_color + 1) - 1
        if degree != int(degree) or not 0 <= degree <= 3:
            raise PlyError(f"Unsupported SH degree: {degree}")
        degree = int(degree)
        self.numGaussians = count
        self.sphericalHarmonicsDegree = degree
        if count >= 2 ** 31:
            raise PlyError("at most 2^31 - 1 vertices")
        # the reference reads float and uchar properties and skips other types
        # without advancing its read offset (src/GS_ply.ts:120-128)
        dtype = [(name, _PLY_TYPES[typ]) for name, typ in props if typ in ("float", "uchar")]
        readable = {name for name, _ in dtype}
        required = (["x", "y", "z", "scale_0", "scale_1", "scale_2", "rot_0", "rot_1", "rot_2", "rot_3", "opacity"]
                    + _sh_feature_order(n_rest))
        for name in required:
            if name not in readable:
                raise PlyError(f"missing float/uchar vertex property {name}")
        dt = np.dtype(dtype)
        if count and offset + dt.itemsize * count > len(buf):
            raise PlyError("PLY vertex data is shorter than the header says")
        rows = np.frombuffer(buf, dtype=dt, count=count, offset=offset)

        def col(name: str) -> np.ndarray:
            v = rows[name].astype(np.float64)
            if dt[name] == np.dtype("u1"):
                v = v / 255.0
            return v

        pos = np.stack([col("x"), col("y"), col("z")], axis=1)
        scale = np.exp(np.stack([col("scale_0"), col("scale_1"), col("scale_2")], axis=1))
        q = np.stack([col(f"rot_{i}") for i in range(4)], axis=1)
        # ((q0^2 + q1^2) + q2^2) + q3^2, the JS expression's order
        norm = np.sqrt(((q[:, 0] * q[:, 0] + q[:, 1] * q[:, 1]) + q[:, 2] * q[:, 2]) + q[:, 3] * q[:, 3])
        q = q / norm[:, None]
        opacity = 1.0 / (1.0 + np.exp(-col("opacity")))
        n_sh = (degree + 1) ** 2
        order = _sh_feature_order(n_rest)
        sh = np.stack([col(nm) for nm in order], axis=1).reshape(count, n_sh, 3)
        self.gaussianData = {"position": pos, "scale": scale, "rotQuat": q,
                             "opacity": opacity, "shCoeffs": sh}
        stride = record_stride(degree)
        rec = np.zeros((count, stride // 4), dtype=np.float32)
        rec[:, 0:3] = pos
        rec[:, 4:7] = scale
        rec[:, 8:12] = q
        rec[:, 12] = opacity
        sh_f = np.zeros((count, n_sh, 4), dtype=np.float32)
        sh_f[:, :, :3] = sh
        rec[:, 16:16 + 4 * n_sh] = sh_f.reshape(count, 4 * n_sh)
        self.gaussiansBuffer = rec
        posb = np.zeros((count, 4), dtype=np.float32)
        posb[:, :3] = pos
        self.positionsBuffer = posb

    def activations(self) -> np.ndarray:
        """(n, 8) float64: opacity, scale xyz, rotation wxyz of gaussianData,
        the values the reference builds its proxies from (src/main.ts:74-87)."""
        d = self.gaussianData
        n = self.numGaussians
        if n == 0:
            return np.zeros((0, 8), dtype=np.float64)
        return np.ascontiguousarray(np.concatenate(
            [np.asarray(d["opacity"], dtype=np.float64).reshape(n, 1), np.asarray(d["scale"], dtype=np.float64),
             np.asarray(d["rotQuat"], dtype=np.float64)], axis=1))

    @property
    def stride_bytes(self) -> int:
        return self.gaussiansBuffer.shape[1] * 4 if self.numGaussians else record_stride(self.sphericalHarmonicsDegree)


def load_gaussian_splatting(path: str) -> PackedGaussians:
    """``loadGaussianSplatting`` (src/GS_ply.ts:4-8) for a local file."""
    with open(path, "rb") as fh:
        return PackedGaussians(fh.read())


PLY_PROPERTIES = (["x", "y", "z", "nx", "ny", "nz", "f_dc_0", "f_dc_1", "f_dc_2"]
                  + [f"f_rest_{i}" for i in range(45)]
                  + ["opacity", "scale_0", "scale_1", "scale_2", "rot_0", "rot_1", "rot_2", "rot_3"])


def write_ply(raw: dict, sh_degree: int = 3) -> bytes:
    """Serialises pre-activation values in the 3DGS PLY layout.

    ``raw`` holds float arrays: ``xyz`` (n,3), ``log_scale`` (n,3),
    ``rot`` (n,4, unnormalised quaternion w,x,y,z), ``opacity_logit`` (n,),
    ``sh`` (n, (deg+1)^2, 3) with sh[:,0] the DC term.
    """
    xyz = np.asarray(raw["xyz"], dtype=np.float32)
    n = xyz.shape[0]
    n_sh = (sh_degree + 1) ** 2
    per_color = n_sh - 1
    names = (["x", "y", "z", "nx", "ny", "nz", "f_dc_0", "f_dc_1", "f_dc_2"]
             + [f"f_rest_{i}" for i in range(3 * per_color)]
             + ["opacity", "scale_0", "scale_1", "scale_2", "rot_0", "rot_1", "rot_2", "rot_3"])
    data = np.zeros((n, len(names)), dtype=np.float32)
    data[:, 0:3] = xyz
    sh = np.asarray(raw["sh"], dtype=np.float32)
    data[:, 6:9] = sh[:, 0, :]
    for c in range(3):
        for i in range(per_color):
            data[:, 9 + c * per_color + i] = sh[:, i + 1, c]
    base = 9 + 3 * per_color
    data[:, base] = np.asarray(raw["opacity_logit"], dtype=np.float32)
    data[:, base + 1:base + 4] = np.asarray(raw["log_scale"], dtype=np.float32)
    data[:, base + 4:base + 8] = np.asarray(raw["rot"], dtype=np.float32)
    header = ["ply", "format binary_little_endian 1.0", f"element vertex {n}"]
    header += [f"property float {nm}" for nm in names]
    header += ["end_header"]
    return ("\n".join(header) + "\n").encode("ascii") + data.astype("<f4").tobytes()
