"""pe_relative_step_noalloc: the relative 5D step for callers that cannot
allocate device memory while they run (a fixed-rate controller that cannot
stall on cudaMalloc/cudaFree, or a host that owns all device memory through
its own pool).  Its scratch lives in a fixed __device__ array inside the
library, so the caller passes only its own input, output and arrival
buffers.

Checked through the C ABI against the existing entry point (a
PE_LOCAL_F64 handle's pe_relative_step) on two calls in a row: the fields
and arrival times must be identical bit for bit.  The CUDA runtime loads
the library's device code lazily, so the first call may reserve the fixed
array (about 16 MB) on the device: that call may take at most the array
plus a module's rounding, and the second call must not change the device's
free memory at all.  This file sorts last so that a run stopping at the
first failure has run every other test first."""

# g_step_scratch in capi_noalloc.cu: stats words, 2 x 1024 heading doubles
# and PE_NOALLOC_MAX_CELLS floats of stage field
SCRATCH_BYTES = 8 * (4 + 2 * 1024) + 4 * 4194304

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_step_without_allocation_equals_handle_step_twice():
    import torch

    from pursuit_evasion_b200 import _native
    from pursuit_evasion_b200.reversible.relative_solver import RelativeSolver, _params
    from tests.helpers import A3, CONFIG1_GRID, CONFIG2_GRID

    lib = _native.library()
    grid = CONFIG1_GRID
    with RelativeSolver(A3, grid, local_precision="float64") as h:
        h.initialize()
        v0, a0 = h.field().ravel().copy(), h.arrival().ravel().copy()
        dt = h.cfl_dt_limit
        h.step(dt)
        v1, a1 = h.field().ravel().copy(), h.arrival().ravel().copy()
        h.step(dt)
        v2, a2 = h.field().ravel().copy(), h.arrival().ravel().copy()

    params = _params(A3, grid, order=2, cfl=0.8, precision=_native.PE_LOCAL_F64,
                     device=0)
    device = torch.device("cuda", 0)
    field_a = torch.from_numpy(v0).to(device)
    field_b = torch.empty_like(field_a)
    arrival = torch.from_numpy(a0).to(device)
    stream = torch.cuda.current_stream(device).cuda_stream
    torch.cuda.synchronize(device)

    residual = ctypes.c_double()
    free_first, _ = torch.cuda.mem_get_info(device)
    rc = lib.pe_relative_step_noalloc(ctypes.byref(params), field_a.data_ptr(),
                                      field_b.data_ptr(), arrival.data_ptr(), 0.0, dt,
                                      stream, ctypes.byref(residual))
    assert rc == 0, lib.pe_last_error()
    np.testing.assert_array_equal(field_b.cpu().numpy().view(np.uint32), v1.view(np.uint32))
    np.testing.assert_array_equal(arrival.cpu().numpy().view(np.uint32), a1.view(np.uint32))
    assert residual.value == np.abs(v1.astype(np.float64) - v0).max()
    free_before, _ = torch.cuda.mem_get_info(device)
    # the first call reserves at most the array (plus 2 MiB pages of the
    # lazily loaded module); nothing when the module was loaded already
    assert 0 <= free_first - free_before <= SCRATCH_BYTES + (8 << 20)

    rc = lib.pe_relative_step_noalloc(ctypes.byref(params), field_b.data_ptr(),
                                      field_a.data_ptr(), arrival.data_ptr(), dt, dt,
                                      stream, None)
    assert rc == 0, lib.pe_last_error()
    free_after, _ = torch.cuda.mem_get_info(device)
    assert free_after == free_before
    np.testing.assert_array_equal(field_a.cpu().numpy().view(np.uint32), v2.view(np.uint32))
    np.testing.assert_array_equal(arrival.cpu().numpy().view(np.uint32), a2.view(np.uint32))

    # A grid above the fixed scratch size is refused before any GPU work.
    big = _params(A3, CONFIG2_GRID, order=2, cfl=0.8, precision=_native.PE_LOCAL_F64,
                  device=0)
    rc = lib.pe_relative_step_noalloc(ctypes.byref(big), field_a.data_ptr(),
                                      field_b.data_ptr(), arrival.data_ptr(), 0.0, dt,
                                      stream, None)
    assert rc == _native.PE_EINVAL
    assert b"at most" in lib.pe_last_error()
