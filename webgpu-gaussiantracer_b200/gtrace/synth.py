"""Seeded synthetic 3DGS scenes and cameras for the benchmark configurations.

The reference ships no benchmark scene (its app loads an absent
``data/train.ply``), so every workload here is generated.  Scenes are made as
pre-activation 3DGS PLY data (log-scale, logit opacity, unnormalised
quaternion) so that the reference's own loader (src/GS_ply.ts:225-235), or
its mirror ``gtrace.ply.PackedGaussians``, produces the stated distributions.

Random streams: numpy ``Generator(PCG64(seed))``; seed = 0x6A5C0000 + config
index (+ a sub-seed per scene or perturbation).

==========  ===================================================================
config      scene / view
==========  ===================================================================
small       16,384 Gaussians; mu ~ N(0,1)^3 clipped to |x| <= 3; log s ~ U[-4.5,-2.5]
            per axis; uniform unit quaternions (Shoemake); opacity ~ U[0.05,0.99];
            SH DC ~ N(0,0.5), bands 1-3 ~ N(0,0.05).  256x256, hFov 60, camera at
            (0,0,4) looking at the origin; alpha_min 0.01, k 6, T_min 0.01
clusters    64 clusters, centres U[-5,5]^3, sigma_c ~ U[0.1,0.8]; mu = c + sigma_c N(0,1)^3;
            log s_x ~ U[-5,-2], log s_y/z = log s_x + U[-ln 10, 0] clipped below at -5;
            opacity = sigmoid(N(0,1.5)); SH as small.  Used by: 1M @ 1920x1080,
            camera radius 12 on +Z, k 16; 200k @ 800x800, k 8; the batched sets.
==========  ===================================================================
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .ply import PackedGaussians, write_ply
from .uniforms import look_at, pack_uniforms

SEED_BASE = 0x6A5C0000


def _rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(seed))


def _shoemake(rng: np.random.Generator, n: int) -> np.ndarray:
    u1, u2, u3 = rng.random(n), rng.random(n), rng.random(n)
    a, b = np.sqrt(1.0 - u1), np.sqrt(u1)
    return np.stack([a * np.sin(2 * math.pi * u2), a * np.cos(2 * math.pi * u2),
                     b * np.sin(2 * math.pi * u3), b * np.cos(2 * math.pi * u3)], axis=1)


def _sh(rng: np.random.Generator, n: int) -> np.ndarray:
    sh = rng.normal(0.0, 0.05, size=(n, 16, 3))
    sh[:, 0, :] = rng.normal(0.0, 0.5, size=(n, 3))
    return sh


def raw_small(n: int = 16384, seed: int = SEED_BASE + 0) -> dict:
    """Pre-activation data of the small uniform scene."""
    rng = _rng(seed)
    xyz = np.clip(rng.normal(0.0, 1.0, size=(n, 3)), -3.0, 3.0)
    log_s = rng.uniform(-4.5, -2.5, size=(n, 3))
    rot = _shoemake(rng, n)
    o = rng.uniform(0.05, 0.99, size=n)
    return {"xyz": xyz, "log_scale": log_s, "rot": rot, "opacity_logit": np.log(o / (1.0 - o)),
            "sh": _sh(rng, n)}


def raw_clusters(n: int, seed: int, n_clusters: int = 64) -> dict:
    """Pre-activation data of the 64-cluster mixture."""
    rng = _rng(seed)
    centres = rng.uniform(-5.0, 5.0, size=(n_clusters, 3))
    sig = rng.uniform(0.1, 0.8, size=n_clusters)
    pick = rng.integers(0, n_clusters, size=n)
    xyz = centres[pick] + sig[pick, None] * rng.normal(0.0, 1.0, size=(n, 3))
    lx = rng.uniform(-5.0, -2.0, size=n)
    ly = np.maximum(lx + rng.uniform(-math.log(10.0), 0.0, size=n), -5.0)
    lz = np.maximum(lx + rng.uniform(-math.log(10.0), 0.0, size=n), -5.0)
    rot = _shoemake(rng, n)
    logit = rng.normal(0.0, 1.5, size=n)
    return {"xyz": xyz, "log_scale": np.stack([lx, ly, lz], axis=1), "rot": rot,
            "opacity_logit": logit, "sh": _sh(rng, n)}


def perturb(raw: dict, seed: int) -> dict:
    """Target scene of the differentiable configs: positions + N(0,0.01),
    opacity logits + N(0,0.1), SH DC + N(0,0.05)."""
    rng = _rng(seed)
    out = {k: np.array(v, copy=True) for k, v in raw.items()}
    n = out["xyz"].shape[0]
    out["xyz"] = out["xyz"] + rng.normal(0.0, 0.01, size=(n, 3))
    out["opacity_logit"] = out["opacity_logit"] + rng.normal(0.0, 0.1, size=n)
    out["sh"][:, 0, :] = out["sh"][:, 0, :] + rng.normal(0.0, 0.05, size=(n, 3))
    return out


def pack(raw: dict) -> PackedGaussians:
    """Runs the raw data through the PLY format and the loader mirror."""
    return PackedGaussians(write_ply(raw))


@dataclass
class View:
    width: int
    height: int
    uniforms: np.ndarray  # 112-byte block


def view(width: int, height: int, position, target=(0.0, 0.0, 0.0), *, k: int, alpha_min: float = 0.01,
         T_min: float = 0.01, hfov: float = 60.0, **kw) -> View:
    u = pack_uniforms(look_at(position, target), width, height, hfov=hfov, t_min=1e-3, t_max=1e5,
                      T_min=T_min, alpha_min=alpha_min, k=k, sh_degree_max=3, **kw)
    return View(width, height, u)


def small_config():
    """16,384 Gaussians, 256x256, k 6, alpha_min 0.01."""
    pg = pack(raw_small())
    return pg, 0.01, view(256, 256, (0.0, 0.0, 4.0), k=6)


def clusters_1m_config(n: int = 1_000_000):
    """1M Gaussians in 64 clusters, 1920x1080, k 16, camera radius 12 on +Z."""
    pg = pack(raw_clusters(n, SEED_BASE + 1))
    return pg, 0.01, view(1920, 1080, (0.0, 0.0, 12.0), k=16)


def clusters_200k_config():
    """200k Gaussians, 800x800, k 8 (the differentiable configuration)."""
    raw = raw_clusters(200_000, SEED_BASE + 3)
    return raw, 0.01, view(800, 800, (0.0, 0.0, 12.0), k=8)


def random_sphere_camera(rng: np.random.Generator, radius_lo: float, radius_hi: float, centre=(0.0, 0.0, 0.0)):
    v = rng.normal(size=3)
    v = v / np.linalg.norm(v)
    r = rng.uniform(radius_lo, radius_hi)
    return tuple(np.asarray(centre) + r * v)


def batched_scenes_config(n_scenes: int = 8, n_views: int = 64, scale: float = 1.0):
    """8 scenes with log-uniform Gaussian counts in [100k, 1M] (times ``scale``),
    64 views round-robin, W ~ U{320..1920}, H ~ U{240..1080}, camera radius
    U[8,14], alpha_min per scene from {0.01, 0.05, 0.1}."""
    rng = _rng(SEED_BASE + 2)
    scenes = []
    for s in range(n_scenes):
        n = int(round(10 ** rng.uniform(5.0, 6.0) * scale))
        a_min = float(rng.choice([0.01, 0.05, 0.1]))
        scenes.append((raw_clusters(max(n, 1), SEED_BASE + 2 + 1000 * (s + 1)), a_min))
    views = []
    for v in range(n_views):
        s = v % n_scenes
        w = int(rng.integers(320, 1921))
        h = int(rng.integers(240, 1081))
        pos = random_sphere_camera(rng, 8.0, 14.0)
        views.append((s, w, h, pos))
    return scenes, views


def batched_fwd_bwd_views(n_views: int = 32):
    """Views of the batched forward + backward configuration over the 1M
    clusters scene: W ~ U{640..1920}, H ~ U{480..1080}, camera radius
    U[10, 14], k 16.  The target scene is ``perturb(raw_clusters(1M,
    SEED_BASE + 1), SEED_BASE + 44)``."""
    rng = _rng(SEED_BASE + 4)
    views = []
    for _ in range(n_views):
        w = int(rng.integers(640, 1921))
        h = int(rng.integers(480, 1081))
        pos = random_sphere_camera(rng, 10.0, 14.0)
        views.append(view(w, h, pos, k=16))
    return views
