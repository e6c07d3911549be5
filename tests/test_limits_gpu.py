"""Failure detection on the GPU without a fault: every device loop of the
trace kernels is bounded, and a ray that reaches a bound stops and reports
it through the status word.  gt_set_limits lowers the bounds so that each
path runs: the call returns GT_ERR_DEVICE_TIMEOUT or GT_ERR_STACK_OVERFLOW
with a message, and the context keeps working afterwards."""
import numpy as np
import pytest

from conftest import small_scene, view
from gtrace import _lib as L
from gtrace._lib import GTraceError
from gtrace.tracer import Scene

pytestmark = pytest.mark.gpu


def _render_status(ctx, scene, v):
    out = np.zeros((v.height, v.width, 4), np.float32)
    u = L.Uniforms.from_buffer_copy(bytes(v.uniforms))
    st = ctx._lib.gt_render(ctx.handle, scene.handle, u, v.width, v.height, out.ctypes.data_as(L.C.c_void_p), 0,
                            None)
    return st, L.last_error(ctx.handle), out


@pytest.mark.parametrize("limits,code", [((1, 0, 0), L.GT_ERR_DEVICE_TIMEOUT), ((0, 2, 0), L.GT_ERR_STACK_OVERFLOW),
                                         ((0, 0, 1), L.GT_ERR_DEVICE_TIMEOUT)])
def test_bounded_loops_report_and_recover(ctx, limits, code):
    pg = small_scene(n=4000, seed=51)
    scene = Scene(ctx, pg.gaussiansBuffer, 0.01)
    v = view(64, 48, k=2)  # k = 2: every ray needs several rounds
    good = ctx.render(scene, v.uniforms, v.width, v.height)
    try:
        ctx.check(ctx._lib.gt_set_limits(ctx.handle, *limits))
        st, msg, _ = _render_status(ctx, scene, v)
        assert st == code, (st, msg)
        assert msg
        # a batch launch and the adjoint see the same limits
        with pytest.raises(GTraceError) as ei:
            ctx.render_batch([(scene, v.uniforms, v.width, v.height)])
        assert ei.value.status == code
    finally:
        ctx.check(ctx._lib.gt_set_limits(ctx.handle, 0, 0, 0))
    again = ctx.render(scene, v.uniforms, v.width, v.height)
    assert np.array_equal(good.view(np.uint32), again.view(np.uint32))
    scene.close()


def test_limit_arguments_checked(ctx):
    assert ctx._lib.gt_set_limits(ctx.handle, 0, 257, 0) == L.GT_ERR_INVALID_ARG
    assert ctx._lib.gt_set_limits(ctx.handle, 0, 0, (1 << 22) + 1) == L.GT_ERR_INVALID_ARG
    assert ctx._lib.gt_set_limits(ctx.handle, 0, 0, 0) == L.GT_OK


def test_out_of_memory_is_an_error_not_a_fault(ctx):
    """A device allocation larger than the GPU returns GT_ERR_OOM (cudaMalloc
    fails cleanly), and the context keeps working."""
    p = L.C.c_void_p()
    st = ctx._lib.gt_device_alloc(ctx.handle, 1 << 50, L.C.byref(p))
    assert st == L.GT_ERR_OOM and not p.value
    assert "memory" in L.last_error(ctx.handle).lower()
    pg = small_scene(n=500, seed=52)
    scene = Scene(ctx, pg.gaussiansBuffer, 0.01)
    v = view(16, 16, k=4)
    ctx.render(scene, v.uniforms, v.width, v.height)
    scene.close()
