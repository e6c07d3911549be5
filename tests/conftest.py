"""Shared fixtures: paths, the gpu marker and scene builders.

Tests marked ``gpu`` need a CUDA device and the built library; the others
run on CPU (oracle, host logic, ABI surface).
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "webgpu-gaussiantracer_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU and the built libgtrace.so")


@pytest.fixture(scope="session")
def ctx():
    from gtrace.tracer import Context
    c = Context(0)
    yield c
    c.close()


def small_scene(n=2048, seed=7):
    """A compact uniform scene (the small config's distributions, fewer particles)."""
    from gtrace import synth
    raw = synth.raw_small(n=n, seed=seed)
    return synth.pack(raw)


def view(w, h, pos=(0.0, 0.0, 4.0), target=(0.0, 0.0, 0.0), **kw):
    from gtrace import synth
    kw.setdefault("k", 6)
    return synth.view(w, h, pos, target, **kw)
