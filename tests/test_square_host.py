"""Legacy 6D square game without a GPU: the table reader against the
reference LocalTable's answers (golden vectors), the host-side C-ABI entry
points against the oracle, and option validation."""

import ctypes
import json

import numpy as np
import pytest

from pursuit_evasion_b200 import _native
from pursuit_evasion_b200.dp.grid import GridSpec, output_times
from pursuit_evasion_b200.dp.native import _params, solve
from pursuit_evasion_b200.dp.table import LocalTable
from pursuit_evasion_b200.model import GameConfig, Vehicle
from tests.helpers import square_goldens

SQUARE = square_goldens()


def config_of(options):
    o = dict(arena=3.0, radius=0.3, vp=1.0, ve=0.3, wp=1.0, we=2.0)
    o.update(options)
    return GameConfig(arena_half_width=o["arena"], capture_radius=o["radius"],
                      pursuer=Vehicle(o["vp"], o["wp"]), evader=Vehicle(o["ve"], o["we"]))


def grid_of(options):
    return GridSpec(options["positions"], options["headings"], options["extent"])


def write_table(folder, options, fields):
    folder.mkdir()
    fields.tofile(folder / "fields.f32")
    (folder / "meta.json").write_text(json.dumps(dict(
        status="complete", history_saved=True,
        tube_projection="min over every internal update, then max with avoid",
        grid=grid_of(options).to_dict(), config=config_of(options).to_dict(),
        times=output_times(options["horizon"], options["output-dt"]).tolist())))


@pytest.mark.parametrize("name", sorted(SQUARE))
def test_local_table_answers_like_the_reference_reader(tmp_path, name):
    z = np.load(SQUARE[name])
    options = json.loads(str(z["options"]))
    write_table(tmp_path / "t", options, z["fields"])
    table = LocalTable(tmp_path / "t")
    np.testing.assert_allclose(table.value(z["query_states"]), z["query_value"],
                               rtol=1e-12, atol=1e-12, equal_nan=True)
    np.testing.assert_allclose(table.field(z["query_states"], z["query_budgets"]),
                               z["query_field"], rtol=1e-12, atol=1e-12, equal_nan=True)


@pytest.mark.parametrize("name", sorted(SQUARE))
def test_host_dt_limit_and_cells_match_the_oracle(oracle, name):
    z = np.load(SQUARE[name])
    options = json.loads(str(z["options"]))
    params = _params(config_of(options), grid_of(options), order=options["order"],
                     cfl=0.8, device=0)
    lib = _native.library()
    dt, cells = ctypes.c_double(), ctypes.c_int64()
    assert lib.pe_square_dt_limit(ctypes.byref(params), ctypes.byref(dt)) == 0
    assert lib.pe_square_cells(ctypes.byref(params), ctypes.byref(cells)) == 0
    cfg = oracle.s6_cfg(options)
    assert dt.value == oracle.lib.po_s6_dt_limit(ctypes.addressof(cfg))
    assert cells.value == grid_of(options).states


@pytest.mark.parametrize("change", [dict(extent=2.5), dict(order=3), dict(cfl=1.5),
                                    dict(positions=4)])
def test_invalid_square_options_are_rejected_before_device_work(change):
    options = dict(positions=7, headings=6, extent=3.5, order=2, cfl=0.8)
    options.update(change)
    params = _native.SquareParams(positions=options["positions"], headings=6,
                                  extent=options["extent"], arena=3.0, capture_radius=0.3,
                                  p_speed=1.0, e_speed=0.3, p_turn_rate=1.0, e_turn_rate=2.0,
                                  cfl=options["cfl"], order=options["order"], device=0)
    handle = ctypes.c_void_p()
    lib = _native.library()
    assert lib.pe_square_create(ctypes.byref(params), ctypes.byref(handle)) == _native.PE_EINVAL
    assert not handle.value


def test_solve_rejects_bad_options_and_existing_output(tmp_path):
    with pytest.raises(ValueError):
        solve(GameConfig(), GridSpec(7, 6, 3.5), tmp_path / "a", horizon=-1.0)
    (tmp_path / "b").mkdir()
    (tmp_path / "b" / "meta.json").write_text("{}")
    with pytest.raises(FileExistsError):
        solve(GameConfig(), GridSpec(7, 6, 3.5), tmp_path / "b")
