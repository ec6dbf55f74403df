"""Compact eight-state semi-Lagrangian contact game on the GPU (pe_compact_*,
pursuit_evasion_b200.local_game.grid_game) against the reference's own
golden vectors (brute-force joint action enumeration, made by
tests/golden/make_compact_golden.py) and the FP64 oracle
(oracle/compact_game.py) on larger random grids.  Tolerances are the
reference's (tests/test_compact_dp.py:69-79): 5e-7 on the capture field,
8e-7 after each backup (float32 field against FP64 enumeration)."""

from pathlib import Path

import numpy as np
import pytest

from pursuit_evasion_b200.local_game.geometry import CircleArena
from pursuit_evasion_b200.local_game.grid_game import (
    PairDomain,
    VehicleGrid,
    backup_gpu,
    backup_packed,
    gpu_arrays,
    initialize_gpu,
    initialize_packed,
    packed_gpu_arrays,
    query_field,
)
from tests.test_compact_oracle import GOLDEN, grids, load_oracle

pytestmark = pytest.mark.gpu

ARENA = CircleArena([], 3)


def vehicle(d):
    n, na = d["allowed"].shape
    return VehicleGrid((), d["states"], np.arange(n, dtype=np.int32), np.zeros((na, 2)),
                       d["successors"], d["weights"], d["allowed"], np.ones((n, na)))


def domain_of(d):
    return PairDomain(d["p_position"], d["lookup"], d["e_indices"], d["counts"],
                      d["offsets"], d["exit_radius"])


def random_grid(n, na, rng, spread=1.0, local=None):
    """Random legal states and 16-vertex stencils (the reference's fake_grid,
    tests/test_compact_dp.py:12-29); `local` draws vertices near the state's
    index instead of anywhere."""
    states = rng.uniform(-spread, spread, (n, 4))
    if local:
        base = np.arange(n)[:, None, None]
        ids = np.clip(base + rng.integers(-local, local + 1, (n, na, 16)), 0, n - 1)
    else:
        ids = rng.integers(n, size=(n, na, 16))
    weights = rng.random((n, na, 16)).astype(np.float32)
    weights[rng.random((n, na, 16)) < 0.2] = 0
    weights /= np.maximum(weights.sum(-1, keepdims=True), 1e-6)
    allowed = rng.random((n, na)) > 0.3
    allowed[:, 0] = True
    return {"states": states, "successors": ids.astype(np.int32),
            "weights": weights.astype(np.float32), "allowed": allowed}


@pytest.mark.parametrize("path", GOLDEN, ids=lambda p: p.stem)
def test_dense_backup_matches_reference_enumeration(path):
    z = np.load(path)
    p, e, _ = grids(z)
    frames = z["frames"]
    radius = float(z["exit_radius"])
    P, E = vehicle(p), vehicle(e)
    a = gpu_arrays(P, E, chunk=2)
    initialize_gpu(a, P, E, ARENA, exit_radius=radius)
    np.testing.assert_allclose(a["current"].get().reshape(frames.shape[1:]), frames[0],
                               atol=5e-7)
    for k in range(1, len(frames)):
        backup_gpu(a, P, E)
        np.testing.assert_allclose(a["current"].get().reshape(frames.shape[1:]), frames[k],
                                   atol=8e-7)
    a.close()


@pytest.mark.parametrize("path", GOLDEN, ids=lambda p: p.stem)
def test_packed_backup_matches_reference_enumeration(path):
    cg = load_oracle()
    z = np.load(path)
    p, e, d = grids(z)
    frames = z["frames"]
    n_p, n_e = frames.shape[1:]
    P, E = vehicle(p), vehicle(e)
    dom = domain_of(d)
    for tiled in (False, True):
        a = packed_gpu_arrays(P, E, dom, chunk=2, tiled_output=tiled)
        initialize_packed(a, P, E, dom, ARENA)
        got = cg.expand_packed(a["current"].get(), d, n_p, n_e, d["exit_radius"])
        np.testing.assert_allclose(got, frames[0], atol=5e-7)
        for k in range(1, len(frames)):
            backup_packed(a, P, E, dom)
            got = cg.expand_packed(a["current"].get(), d, n_p, n_e, d["exit_radius"])
            np.testing.assert_allclose(got, frames[k], atol=8e-7)
        a.close()


@pytest.mark.parametrize("n_p, n_e, na_p, na_e, local", [
    (300, 420, 9, 9, None),
    (257, 513, 9, 9, 40),
    (3, 50_000, 9, 3, 500),  # a pursuer row longer than shared memory
])
def test_dense_backup_matches_oracle_on_random_grids(n_p, n_e, na_p, na_e, local):
    cg = load_oracle()
    rng = np.random.default_rng(n_p * 1000 + n_e)
    p = random_grid(n_p, na_p, rng, local=local)
    e = random_grid(n_e, na_e, rng, local=local)
    radius = 1.1
    P, E = vehicle(p), vehicle(e)
    a = gpu_arrays(P, E)
    initialize_gpu(a, P, E, ARENA, exit_radius=radius)
    field = a["current"].get().reshape(n_p, n_e).astype(np.float64)
    ref = cg.capture_field(p["states"], e["states"], (0.8, 0.5), (0.4, 0.25), radius)
    np.testing.assert_allclose(field, ref, atol=5e-7)
    for _ in range(3):
        expected = cg.backup_dense(field, p, e, radius)
        backup_gpu(a, P, E)
        field = a["current"].get().reshape(n_p, n_e).astype(np.float64)
        np.testing.assert_allclose(field, expected, atol=1e-6)
        assert np.all(field <= ref + 1e-6)  # the backup never raises a value
    a.close()


def test_packed_backup_and_query_match_oracle_on_a_random_grid():
    cg = load_oracle()
    rng = np.random.default_rng(5)
    n_p, n_e = 180, 240
    p = random_grid(n_p, 9, rng, spread=2.0, local=30)
    e = random_grid(n_e, 9, rng, spread=2.0, local=30)
    p["states"][:, :2] = np.round(p["states"][:, :2] * 2) / 2  # shared positions
    P, E = vehicle(p), vehicle(e)
    dom = PairDomain.build(P, E, 1.5)
    d = {k: getattr(dom, k) for k in ("p_position", "lookup", "e_indices", "counts", "offsets")}
    d["exit_radius"] = dom.exit_radius
    a = packed_gpu_arrays(P, E, dom)
    initialize_packed(a, P, E, dom, ARENA)
    flat = a["current"].get().astype(np.float64)
    for _ in range(3):
        expected = cg.backup_packed(flat, p, e, d)
        backup_packed(a, P, E, dom)
        flat = a["current"].get().astype(np.float64)
        np.testing.assert_allclose(flat, expected, atol=1e-6)
    n = 500
    pi = rng.integers(n_p, size=(n, 16)).astype(np.int32)
    ei = rng.integers(n_e, size=(n, 16)).astype(np.int32)
    pw = (rng.random((n, 16)) * (rng.random((n, 16)) > 0.4)).astype(np.float32)
    ew = (rng.random((n, 16)) * (rng.random((n, 16)) > 0.4)).astype(np.float32)
    got = query_field(a, pi, pw, ei, ew)
    want = cg.query_packed(flat, pi, pw, ei, ew, d, n_e)
    np.testing.assert_allclose(got, want, rtol=1e-5, atol=1e-5)
    a.close()


def test_device_field_is_zero_copy_viewable():
    import torch

    z = np.load(GOLDEN[0])
    p, e, _ = grids(z)
    P, E = vehicle(p), vehicle(e)
    a = gpu_arrays(P, E)
    initialize_gpu(a, P, E, ARENA, exit_radius=float(z["exit_radius"]))
    view = torch.as_tensor(a["current"], device="cuda")
    np.testing.assert_array_equal(view.cpu().numpy(), a["current"].get())
    a.close()


def test_memory_guard_raises_before_allocating():
    z = np.load(GOLDEN[0])
    p, e, _ = grids(z)
    with pytest.raises(MemoryError):
        gpu_arrays(vehicle(p), vehicle(e), max_gb=1e-9)


def test_grouped_actions_carry_the_running_minimum():
    """A reach list of 20,000 evader states leaves shared memory for only a
    few pursuer actions per pass; with the first actions disallowed for some
    states, later passes start from the minimum of earlier ones (or from the
    current value when no earlier pass ran)."""
    cg = load_oracle()
    rng = np.random.default_rng(21)
    p = random_grid(5, 9, rng, spread=0.3, local=2)
    e = random_grid(20_000, 4, rng, spread=0.3, local=300)
    p["allowed"][:3, :4] = False
    p["allowed"][:3, 8] = True
    radius = 1.0
    P, E = vehicle(p), vehicle(e)
    a = gpu_arrays(P, E)
    initialize_gpu(a, P, E, ARENA, exit_radius=radius)
    field = a["current"].get().reshape(5, 20_000).astype(np.float64)
    for _ in range(2):
        expected = cg.backup_dense(field, p, e, radius)
        backup_gpu(a, P, E)
        field = a["current"].get().reshape(5, 20_000).astype(np.float64)
        np.testing.assert_allclose(field, expected, atol=1e-6)
    a.close()
