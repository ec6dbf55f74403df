"""The C ABI without a GPU: the library loads, exports every symbol that
include/pe_b200.h declares, and its host-only entry points agree with the
oracle; invalid options fail with PE_EINVAL and a message."""

import ctypes
import re
from pathlib import Path

import pytest

from pursuit_evasion_b200 import _native
from pursuit_evasion_b200.reversible.relative_solver import _params
from tests.helpers import A3, CONFIG1_GRID, CONFIG2_GRID, DEFAULT
from pursuit_evasion_b200.reversible.free_dp import RelativeGrid

HEADER = Path(__file__).resolve().parents[1] / "include" / "pe_b200.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pe_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _native.library()
    names = declared_functions()
    assert "pe_relative_create" in names and len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python binding types every one of them
    assert not set(names) - set(_native.SIGNATURES)


def test_version_and_launch_counter():
    lib = _native.library()
    assert lib.pe_version() == 1
    assert lib.pe_launch_count() >= 0


@pytest.mark.parametrize("config,grid", [(A3, CONFIG1_GRID), (A3, CONFIG2_GRID),
                                         (DEFAULT, RelativeGrid(9, 8, 7, 7, 1.0))])
def test_host_cfl_limit_matches_oracle_bitwise(oracle, config, grid):
    lib = _native.library()
    params = _params(config, grid, order=2, cfl=0.8, precision=0, device=0)
    out = ctypes.c_double()
    assert lib.pe_relative_cfl_limit(ctypes.byref(params), ctypes.byref(out)) == 0
    assert out.value == oracle.rel_cfl_limit(oracle.rel_cfg(config, grid))
    cells = ctypes.c_int64()
    assert lib.pe_relative_cells(ctypes.byref(params), ctypes.byref(cells)) == 0
    assert cells.value == grid.states


@pytest.mark.parametrize("field,value", [("positions", 2), ("headings", 3),
                                         ("order", 3), ("cfl", 1.5),
                                         ("capture_radius", 5.0),
                                         ("p_acceleration", 0.0),
                                         ("precision", 7)])
def test_invalid_options_are_rejected_before_any_device_work(field, value):
    lib = _native.library()
    params = _params(A3, CONFIG1_GRID, order=2, cfl=0.8, precision=0, device=0)
    setattr(params, field, value)
    handle = ctypes.c_void_p()
    rc = lib.pe_relative_create(ctypes.byref(params), ctypes.byref(handle))
    assert rc == _native.PE_EINVAL
    assert handle.value is None
    assert b"Invalid" in lib.pe_last_error() or b"unknown" in lib.pe_last_error()
    with pytest.raises(ValueError):
        _native.check(rc)


def test_null_handle_calls_fail_cleanly():
    lib = _native.library()
    assert lib.pe_relative_advance(None, 1.0, None) == _native.PE_EINVAL
    assert lib.pe_relative_destroy(None) == 0


def _compact_grid(n, na, rng, bad_id=False):
    import numpy as np

    pose = rng.uniform(-1, 1, (n, 4)).astype(np.float32)
    ids = rng.integers(n, size=(n, na, 16)).astype(np.int32)
    w = np.full((n, na, 16), 1 / 16, np.float32)
    if bad_id:
        ids[0, 0, 3] = n  # out of range with a positive weight
    allowed = np.ones((n, na), np.uint8)
    keep = [pose, ids, w, allowed]
    return _native.VehicleGridArrays(n, na, *(a.ctypes.data for a in keep)), keep


@pytest.mark.parametrize("case", ["bad_vertex", "radius", "no_actions", "domain"])
def test_compact_create_rejects_invalid_grids_before_device_work(case):
    """pe_compact_create validates grids, radius and pair domain on the host
    (no CUDA call is made before the checks)."""
    import numpy as np

    lib = _native.library()
    rng = np.random.default_rng(0)
    p, keep_p = _compact_grid(5, 3, rng, bad_id=case == "bad_vertex")
    e, keep_e = _compact_grid(7, 4, rng)
    if case == "no_actions":
        e.actions = 0
    radius = -1.0 if case == "radius" else 1.2
    dom = None
    keep_d = []
    if case == "domain":
        lookup = np.full((1, 7), -1, np.int32)
        lookup[0, 2] = 0
        arrays = [np.zeros(5, np.int32), lookup, np.array([[3]], np.int32),
                  np.array([1], np.int32), np.arange(6, dtype=np.int64)]
        keep_d = arrays  # e_indices says 3 but lookup says 2: inconsistent
        dom = ctypes.byref(_native.PairDomainArrays(1, 1, *(a.ctypes.data for a in arrays)))
    handle = ctypes.c_void_p()
    rc = lib.pe_compact_create(ctypes.byref(p), ctypes.byref(e), dom, radius, 0,
                               ctypes.byref(handle))
    assert rc == _native.PE_EINVAL
    assert lib.pe_last_error()
    assert not handle.value
    del keep_p, keep_e, keep_d
