"""Allocation-free grid build (smr_build_grid_static) vs the allocating smr_build_grid (needs a GPU).

smr_build_grid_static serves callers that cannot call cudaMalloc: a host that owns all device
memory through its own pool and forbids allocation after start-up.  It keeps its scratch in one
static device array shared by every call, so this test makes two calls in a row with different
slabs and grid shapes and checks each against the allocating entry point, with the tolerance of
the grid-build parity test, then repeats a build on a caller-owned non-default stream that is
synchronised only through that stream.  The output buffers are allocated by the test (the
caller), as such callers would from their own pools.
"""
import ctypes as C

import numpy as np
import pytest

from surfmol_b200 import synth

pytestmark = pytest.mark.gpu


def _static_build(L, native, slab, dims, p0, step, stream=None):
    """One call on `stream` (a torch.cuda.Stream; None: the current stream), then a wait on that
    stream alone before the result is read."""
    import torch
    nx, ny, nz = dims
    st = stream if stream is not None else torch.cuda.current_stream()
    with torch.cuda.stream(st):
        out = torch.zeros(nx * ny * nz * 4, dtype=torch.float32, device="cuda")
    ions = np.ascontiguousarray(slab.ions, dtype=np.float64)
    re = np.ascontiguousarray(slab.req()[:, :2], dtype=np.float64)
    prm = native.SmrGridBuildParamsStatic(1.5, 1, 1e-12, 0, 0.0)
    err = C.create_string_buffer(256)
    r = L.smr_build_grid_static(len(ions), ions.ctypes.data_as(native.DP), re.ctypes.data_as(native.DP), slab.Lx, slab.Ly,
                                nx, ny, nz, np.asarray(p0, np.float64).ctypes.data_as(native.DP),
                                np.asarray(step, np.float64).ctypes.data_as(native.DP), C.byref(prm),
                                C.c_void_p(out.data_ptr()), C.c_void_p(st.cuda_stream), err, 256)
    assert r == 0, err.value.decode()
    st.synchronize()
    with torch.cuda.stream(st):
        host = out.cpu().numpy().reshape(nx, ny, nz, 4)
    return host


def test_static_grid_build_matches_allocating_build(native):
    from surfmol_b200 import RelaxMulti
    L = native.lib()
    R = RelaxMulti(max_systems=4, max_atoms=64)
    try:
        cases = [(synth.rocksalt_slab(1, 2), (28, 28, 48), 0.2), (synth.rocksalt_slab(2, 3), (40, 36, 30), 0.25)]
        for slab, dims, dz in cases:              # two calls in a row through the shared static scratch
            step = (slab.Lx / dims[0], slab.Ly / dims[1], dz)
            p0 = (0.0, 0.0, slab.z_top + 1.0)
            R.build_grid(slab.ions, slab.req()[:, :2], slab.Lx, slab.Ly, dims[0], dims[1], dims[2], p0, step)
            ref = R.get_grid()["coef"].astype(np.float64)
            got = _static_build(L, native, slab, dims, p0, step).astype(np.float64)
            for c in range(3):
                scale = np.abs(ref[..., c]).max()
                assert np.abs(got[..., c] - ref[..., c]).max() < 2e-6 * scale, c
            assert np.all(got[..., 3] == 0)
        # the same build on a fresh caller-owned stream, waited for through that stream only
        import torch
        slab, dims, dz = cases[0]
        step = (slab.Lx / dims[0], slab.Ly / dims[1], dz)
        p0 = (0.0, 0.0, slab.z_top + 1.0)
        R.build_grid(slab.ions, slab.req()[:, :2], slab.Lx, slab.Ly, dims[0], dims[1], dims[2], p0, step)
        ref = R.get_grid()["coef"].astype(np.float64)
        got = _static_build(L, native, slab, dims, p0, step, stream=torch.cuda.Stream()).astype(np.float64)
        for c in range(3):
            assert np.abs(got[..., c] - ref[..., c]).max() < 2e-6 * np.abs(ref[..., c]).max(), c
    finally:
        R.finish()


def test_static_grid_build_rejects_oversize(native):
    import torch
    L = native.lib()
    slab = synth.rocksalt_slab(1, 2)
    out = torch.zeros(4, dtype=torch.float32, device="cuda")
    prm = native.SmrGridBuildParamsStatic(1.5, 1, 1e-12, 0, 0.0)
    err = C.create_string_buffer(256)
    ions = np.ascontiguousarray(slab.ions)
    re = np.ascontiguousarray(slab.req()[:, :2])
    p0 = np.array([0.0, 0.0, 1.0])
    step = np.array([0.05, 0.05, 0.05])
    r = L.smr_build_grid_static(len(ions), ions.ctypes.data_as(native.DP), re.ctypes.data_as(native.DP), slab.Lx, slab.Ly,
                                400, 400, 400, p0.ctypes.data_as(native.DP), step.ctypes.data_as(native.DP), C.byref(prm),
                                C.c_void_p(out.data_ptr()), None, err, 256)
    assert r == -3 and b"scratch" in err.value
