"""The allocation-free interior step, for callers that cannot call cudaMalloc
where they step the field (real-time callbacks that must not block on the
allocator, hosts whose memory pool owns the free HBM).

It is checked through the C-ABI against the library's own FP64 step on the
non-PML cells of a source-free, body-free solve, on two calls in a row.  This
file is collected last so that a failure here leaves every other test run.
"""
import ctypes as C

import numpy as np
import pytest

from acoustics_b200 import scene as S
from acoustics_b200._lib import load
from acoustics_b200.solver import PML_WaveSolver

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-12


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def test_noalloc_interior_step_matches_solver_on_two_calls():
    import torch

    lib = load()
    h = 0.005
    dims = (40, 36, 44)
    sc = S.Scene(cell_size=h, divisions=dims, time_step=S.reference_time_step(h), pml_width=6)
    sc.sources.append(S.GaussianSource((0.012, -0.006, 0.01), 2e-5))
    sc.listeners = np.array([[0.0, 0.0, 0.0]])
    g = PML_WaveSolver(sc)
    # past the source window: |t + k/2 - t0| / sigma_t > 40 after 190 steps
    g.step(200)
    W = 6
    lo = (C.c_int32 * 3)(W, W, W)
    hi = (C.c_int32 * 3)(*[n - W for n in dims])
    cdims = (C.c_int32 * 3)(*dims)
    box = tuple(slice(W, n - W) for n in dims)
    c2k2 = (sc.sound_speed * sc.time_step) * (sc.sound_speed * sc.time_step)
    lap_scale = 1.0 / (h * h)

    p_cur = torch.tensor(g.field(S.FIELD_PRESSURE), dtype=torch.float64, device="cuda")
    p_prev = torch.tensor(g.field(S.FIELD_PRESSURE_PREV), dtype=torch.float64, device="cuda")
    assert float(p_cur.abs().max()) > 0.0
    for call in range(2):
        p_next = torch.zeros_like(p_cur)
        st = lib.fdtd_interior_step_noalloc(C.c_void_p(p_cur.data_ptr()), C.c_void_p(p_prev.data_ptr()),
                                            C.c_void_p(p_next.data_ptr()), cdims, lo, hi, c2k2, lap_scale, None)
        assert st == 0, lib.fdtd_last_error()
        torch.cuda.synchronize()
        g.step(1)
        ref = g.field(S.FIELD_PRESSURE).reshape(dims)[box]
        got = p_next.cpu().numpy().reshape(dims)[box]
        assert np.abs(ref).max() > 0.0
        assert _rel(got, ref) <= TOL_FP64, call
        # cells outside the box are not written
        outside = np.ones(dims, dtype=bool)
        outside[box] = False
        assert np.all(p_next.cpu().numpy().reshape(dims)[outside] == 0.0)
        # the next call needs p^{n+1} on the PML cells around the box too: take them
        # from the library's step, keep this entry point's values inside the box
        full = torch.tensor(g.field(S.FIELD_PRESSURE), dtype=torch.float64, device="cuda").reshape(dims)
        full[box] = p_next.reshape(dims)[box]
        p_prev, p_cur = p_cur, full.reshape(-1).contiguous()
    g.close()


def test_noalloc_in_place_equals_separate_output():
    """p_next may be p_prev: the step written over p^{n-1} equals the step written
    into a separate buffer, on two calls in a row."""
    import torch

    lib = load()
    dims = (36, 40, 44)
    g = torch.Generator().manual_seed(3)
    p_cur = torch.rand(dims, generator=g, dtype=torch.float64).reshape(-1).cuda()
    p_prev = torch.rand(dims, generator=g, dtype=torch.float64).reshape(-1).cuda()
    cdims = (C.c_int32 * 3)(*dims)
    lo = (C.c_int32 * 3)(2, 3, 1)
    hi = (C.c_int32 * 3)(30, 37, 41)
    c2k2, lap_scale = 0.08, 1.0
    for call in range(2):
        sep = torch.zeros_like(p_cur)
        st = lib.fdtd_interior_step_noalloc(C.c_void_p(p_cur.data_ptr()), C.c_void_p(p_prev.data_ptr()),
                                            C.c_void_p(sep.data_ptr()), cdims, lo, hi, c2k2, lap_scale, None)
        assert st == 0, lib.fdtd_last_error()
        inplace = p_prev.clone()
        st = lib.fdtd_interior_step_noalloc(C.c_void_p(p_cur.data_ptr()), C.c_void_p(inplace.data_ptr()),
                                            C.c_void_p(inplace.data_ptr()), cdims, lo, hi, c2k2, lap_scale, None)
        assert st == 0, lib.fdtd_last_error()
        torch.cuda.synchronize()
        box = tuple(slice(lo[d], hi[d]) for d in range(3))
        a = sep.cpu().numpy().reshape(dims)[box]
        b = inplace.cpu().numpy().reshape(dims)[box]
        assert np.array_equal(a, b), call
        # outside the box the in-place buffer keeps p^{n-1}
        outside = np.ones(dims, dtype=bool)
        outside[box] = False
        assert np.array_equal(inplace.cpu().numpy().reshape(dims)[outside], p_prev.cpu().numpy().reshape(dims)[outside])
        p_prev, p_cur = p_cur, inplace


def test_noalloc_rejects_boxes_beyond_the_scratch_limit():
    lib = load()
    import torch
    n = 130                                  # 128^3 box > FDTD_NOALLOC_MAX_CELLS = 2^20
    buf = torch.zeros(1, dtype=torch.float64, device="cuda")
    cdims = (C.c_int32 * 3)(n, n, n)
    lo = (C.c_int32 * 3)(1, 1, 1)
    hi = (C.c_int32 * 3)(n - 1, n - 1, n - 1)
    p = C.c_void_p(buf.data_ptr())
    st = lib.fdtd_interior_step_noalloc(p, p, p, cdims, lo, hi, 0.1, 1.0, None)
    assert st == -1
    assert b"FDTD_NOALLOC_MAX_CELLS" in lib.fdtd_last_error()
    bad_lo = (C.c_int32 * 3)(0, 1, 1)
    st = lib.fdtd_interior_step_noalloc(p, p, p, cdims, bad_lo, hi, 0.1, 1.0, None)
    assert st == -1
