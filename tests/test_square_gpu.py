"""Legacy 6D square game on the GPU (pe_square_*, pursuit_evasion_b200.dp)
against the reference executable native_square.cpp: its golden frames bit
for bit, its own output folder when the executable is built, and the table
reader on the GPU's fields."""

import json
import shutil
import subprocess

import numpy as np
import pytest

from pursuit_evasion_b200.dp.native import SquareSolver, solve
from pursuit_evasion_b200.dp.table import LocalTable
from tests import oracle_lib
from tests.helpers import bits, square_goldens
from tests.test_square_host import config_of, grid_of

pytestmark = pytest.mark.gpu

SQUARE = square_goldens()
REF_SQUARE = oracle_lib.ORACLE_DIR / "_ref" / "square6d"


@pytest.mark.parametrize("name", sorted(SQUARE))
def test_square_solver_reproduces_reference_golden_bitwise(name):
    z = np.load(SQUARE[name])
    options = json.loads(str(z["options"]))
    with SquareSolver(config_of(options), grid_of(options), order=options["order"]) as s:
        s.initialize()
        frames = [s.field().copy()]
        horizon, out_dt = options["horizon"], options["output-dt"]
        for frame in range(1, int(np.ceil(horizon / out_dt - 1e-10)) + 1):
            s.advance(min(horizon, frame * out_dt))
            frames.append(s.field().copy())
        assert s.steps == int(z["internal_steps"])
        np.testing.assert_array_equal(bits(np.array(frames)), bits(z["fields"]))
        np.testing.assert_array_equal(bits(s.arrival().ravel()), bits(z["arrival"]))


@pytest.mark.parametrize("name", sorted(SQUARE))
def test_solve_writes_the_reference_table(tmp_path, name):
    z = np.load(SQUARE[name])
    options = json.loads(str(z["options"]))
    meta = solve(config_of(options), grid_of(options), tmp_path / "s",
                 horizon=options["horizon"], output_dt=options["output-dt"],
                 order=options["order"])
    assert meta["status"] == "complete" and meta["internal_steps"] == int(z["internal_steps"])
    for key, file in (("fields", "fields.f32"), ("final", "final.f32"),
                      ("arrival", "arrival.f32")):
        np.testing.assert_array_equal(np.fromfile(tmp_path / "s" / file, np.uint32),
                                      bits(z[key]).ravel(), err_msg=file)
    table = LocalTable(tmp_path / "s")
    np.testing.assert_allclose(table.value(z["query_states"]), z["query_value"],
                               rtol=1e-12, atol=1e-12, equal_nan=True)


@pytest.mark.skipif(not REF_SQUARE.exists(),
                    reason="reference executable not built (make -C oracle ref)")
def test_default_grid_matches_the_reference_executable(tmp_path):
    """The reference's default grid (17 positions, 16 headings, 21.4M cells)
    for 0.2 s: same final field and arrival as the executable itself."""
    out = tmp_path / "ref"
    subprocess.run([str(REF_SQUARE), "--horizon", "0.2", "--output-dt", "0.1", "--threads",
                    "8", "--history", "0", "--output", str(out)], check=True,
                   capture_output=True)
    meta = solve(config_of({}), grid_of(dict(positions=17, headings=16, extent=3.5)),
                 tmp_path / "gpu", horizon=0.2, output_dt=0.1, history=False)
    timing = json.loads((out / "native_timing.json").read_text())
    assert meta["internal_steps"] == timing["internal_steps"]
    for file in ("final.f32", "arrival.f32"):
        np.testing.assert_array_equal(np.fromfile(tmp_path / "gpu" / file, np.uint32),
                                      np.fromfile(out / file, np.uint32), err_msg=file)
    shutil.rmtree(out)
