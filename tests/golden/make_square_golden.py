"""Generate the legacy 6D square-game golden vectors from the REFERENCE
executable itself (src/pursuit_evasion/dp/native_square.cpp, compiled from
the reference sources by `make -C oracle ref` into oracle/_ref/square6d with
the reference's own flags, dp/native.py:45-49).

    square6d_<name>.npz   every frame of fields.f32, final.f32, arrival.f32,
                          native_timing.json's internal_steps and
                          max_internal_dt, and the options used

Run in a container where the reference tree is mounted:
    make -C oracle ref && python tests/golden/make_square_golden.py
"""

import json
from pathlib import Path
import subprocess
import tempfile

import numpy as np

HERE = Path(__file__).resolve().parent
EXE = HERE.parents[1] / "oracle" / "_ref" / "square6d"

# name -> executable options (the reference's defaults for the rest:
# arena 3, radius 0.3, vp 1, ve 0.3, wp 1, we 2, cfl 0.8)
CASES = {
    "7x6_o2": dict(positions=7, headings=6, extent=3.5, horizon=0.6, **{"output-dt": 0.2},
                   order=2),
    "7x6_o1": dict(positions=7, headings=6, extent=3.5, horizon=0.2, **{"output-dt": 0.1},
                   order=1),
    "9x4_o2_fast_e": dict(positions=9, headings=4, extent=4.0, arena=3.0, radius=0.5,
                          vp=1.2, ve=0.8, wp=1.5, we=2.5, horizon=0.25,
                          **{"output-dt": 0.125}, order=2),
}


def run(options):
    with tempfile.TemporaryDirectory(dir=HERE) as tmp:
        out = Path(tmp) / "out"
        cmd = [str(EXE)] + [str(v) for k, x in options.items() for v in ("--" + k, x)]
        cmd += ["--threads", "2", "--history", "1", "--output", str(out)]
        subprocess.run(cmd, check=True, capture_output=True)
        timing = json.loads((out / "native_timing.json").read_text())
        n, h = options["positions"], options["headings"]
        shape = (n, n, h, n, n, h)
        fields = np.fromfile(out / "fields.f32", np.float32).reshape(-1, *shape)
        return dict(fields=fields, final=np.fromfile(out / "final.f32", np.float32),
                    arrival=np.fromfile(out / "arrival.f32", np.float32),
                    internal_steps=timing["internal_steps"],
                    max_internal_dt=timing["max_internal_dt"])


def reference_queries(options, r, tmp):
    """value() and field() of the reference's LocalTable (dp/table.py:17-123,
    imported read-only from the reference tree) on the executable's fields,
    at seeded random states."""
    import os
    import sys

    sys.path.insert(0, os.path.join(os.environ.get("PE_REFERENCE_ROOT", "/root/reference"),
                                    "src"))
    from pursuit_evasion.dp.grid import GridSpec, output_times
    from pursuit_evasion.dp.table import LocalTable
    from pursuit_evasion.model import GameConfig, Vehicle

    o = dict(arena=3.0, radius=0.3, vp=1.0, ve=0.3, wp=1.0, we=2.0)
    o.update(options)
    config = GameConfig(arena_half_width=o["arena"], capture_radius=o["radius"],
                        pursuer=Vehicle(o["vp"], o["wp"]), evader=Vehicle(o["ve"], o["we"]))
    grid = GridSpec(options["positions"], options["headings"], options["extent"])
    folder = Path(tmp) / "table"
    folder.mkdir()
    r["fields"].tofile(folder / "fields.f32")
    (folder / "meta.json").write_text(json.dumps(dict(
        status="complete", history_saved=True,
        tube_projection="min over every internal update, then max with avoid",
        grid=grid.to_dict(), config=config.to_dict(),
        times=output_times(options["horizon"], options["output-dt"]).tolist())))
    table = LocalTable(folder)
    rng = np.random.default_rng(6)
    e = options["extent"]
    states = np.concatenate([rng.uniform(-e * 1.05, e * 1.05, (64, 6)),
                             rng.uniform(-2.0, 2.0, (64, 6))])
    states[:, [2, 5]] = rng.uniform(-4, 4, (128, 2))
    budgets = rng.uniform(0, options["horizon"], 128)
    return dict(query_states=states, query_budgets=budgets,
                query_value=table.value(states), query_field=table.field(states, budgets))


def main():
    for name, options in CASES.items():
        r = run(options)
        with tempfile.TemporaryDirectory(dir=HERE) as tmp:
            r.update(reference_queries(options, r, tmp))
        np.savez_compressed(HERE / f"square6d_{name}.npz", options=json.dumps(options), **r)
        print(name, r["fields"].shape, r["internal_steps"],
              int(np.isfinite(r["query_value"]).sum()), "finite values")


if __name__ == "__main__":
    main()
