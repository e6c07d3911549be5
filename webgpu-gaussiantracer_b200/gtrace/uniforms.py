"""The 112-byte uniform block and the camera convention of the reference.

``pack_uniforms`` mirrors ``upadateUniformData`` (src/main.ts:516-534) and
produces the block the ray-generation shader reads (src/GS_shader.ts:96-108):

====  ========================  ==========================================
byte  field                     value
====  ========================  ==========================================
0     toWorld mat4              camera matrix, column-major (right, up, back,
                                position), as camera.matrix (src/camera.ts:11-21)
64    cameraAspect vec2         tan(hFov/2) and that f32 value times H/W
72    t_min, 76 t_max           ray interval
80    T_min                     transmittance cutoff
84    alpha_min                 compositing threshold
88    k (u32)                   hit_array_size
92    sh_degree_max (u32)
96    accumulatedFrames (u32)
100   earlyStop (u32)           earlyStop <= 0 -> 0xFFFFFFFF (off)
104   debugMode (u32)
====  ========================  ==========================================

``look_at`` builds the matrix of ``WASDCamera`` after its first update
(src/camera.ts:122-190): yaw = atan2(back.x, back.z), pitch = -asin(back.y)
with back = normalize(position - target), rotation = rotY(yaw) * rotX(pitch).
"""
from __future__ import annotations

import math

import numpy as np

UNIFORM_BYTES = 112


def look_at(position, target=(0.0, 0.0, 0.0)) -> np.ndarray:
    """Column-major 4x4 camera matrix (float32, 16 values)."""
    p = np.asarray(position, dtype=np.float64)
    t = np.asarray(target, dtype=np.float64)
    back = p - t
    back = back / np.linalg.norm(back)
    yaw = math.atan2(back[0], back[2])
    pitch = -math.asin(max(-1.0, min(1.0, back[1])))
    cy, sy = math.cos(yaw), math.sin(yaw)
    cp, sp = math.cos(pitch), math.sin(pitch)
    ry = np.array([[cy, 0, sy], [0, 1, 0], [-sy, 0, cy]])
    rx = np.array([[1, 0, 0], [0, cp, -sp], [0, sp, cp]])
    r = ry @ rx
    m = np.eye(4)
    m[:3, :3] = r
    m[:3, 3] = p
    return m.T.reshape(16).astype(np.float32)  # column-major


def pack_uniforms(to_world, width: int, height: int, *, hfov: float = 60.0, t_min: float = 1e-3,
                  t_max: float = 1e5, T_min: float = 0.03, alpha_min: float = 0.2, k: int = 6,
                  sh_degree_max: int = 3, accumulated_frames: int = 0, early_stop: int = 0,
                  debug_mode: int = 0) -> np.ndarray:
    """Returns the 112-byte block as a uint8 array (defaults: src/main.ts:448-464)."""
    buf = np.zeros(UNIFORM_BYTES, dtype=np.uint8)
    f = buf.view(np.float32)
    u = buf.view(np.uint32)
    f[0:16] = np.asarray(to_world, dtype=np.float32).reshape(16)
    f[16] = np.float32(math.tan(0.5 * hfov * math.pi / 180.0))
    f[17] = np.float32(float(f[16]) * (height / width))
    f[18] = t_min
    f[19] = t_max
    f[20] = T_min
    f[21] = alpha_min
    u[22] = k
    u[23] = sh_degree_max
    u[24] = accumulated_frames
    u[25] = 0xFFFFFFFF if early_stop <= 0 else early_stop
    u[26] = debug_mode
    return buf


def unpack_uniforms(buf) -> dict:
    b = np.frombuffer(bytes(buf), dtype=np.uint8)
    f = b.view(np.float32)
    u = b.view(np.uint32)
    return {"to_world": f[0:16].copy(), "camera_aspect": f[16:18].copy(), "t_min": float(f[18]),
            "t_max": float(f[19]), "T_min": float(f[20]), "alpha_min": float(f[21]), "k": int(u[22]),
            "sh_degree_max": int(u[23]), "accumulated_frames": int(u[24]), "early_stop": int(u[25]),
            "debug_mode": int(u[26])}


def with_fields(buf, **changes) -> np.ndarray:
    """Copy of a uniform block with some u32/f32 fields replaced."""
    out = np.frombuffer(bytes(buf), dtype=np.uint8).copy()
    f = out.view(np.float32)
    u = out.view(np.uint32)
    fmap = {"t_min": 18, "t_max": 19, "T_min": 20, "alpha_min": 21}
    umap = {"k": 22, "sh_degree_max": 23, "accumulated_frames": 24, "early_stop": 25, "debug_mode": 26}
    for key, val in changes.items():
        if key in fmap:
            f[fmap[key]] = val
        elif key in umap:
            u[umap[key]] = val
        else:
            raise KeyError(key)
    return out
