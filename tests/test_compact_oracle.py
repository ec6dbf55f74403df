"""The compact 8D semi-Lagrangian oracle (oracle/compact_game.py) against
golden vectors produced by the reference's own test helpers
(tests/golden/make_compact_golden.py)."""

import importlib.util
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parents[1]
GOLDEN = sorted((REPO / "tests" / "golden").glob("compact8d_*.npz"))


def load_oracle():
    spec = importlib.util.spec_from_file_location(
        "compact_game_oracle", REPO / "oracle" / "compact_game.py")
    module = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(module)
    return module


def grids(z):
    p = {k: z["p_" + k] for k in ("states", "successors", "weights", "allowed")}
    e = {k: z["e_" + k] for k in ("states", "successors", "weights", "allowed")}
    domain = {k: z[k] for k in ("p_position", "lookup", "e_indices", "counts", "offsets")}
    domain["exit_radius"] = float(z["exit_radius"])
    return p, e, domain


@pytest.fixture(scope="module")
def cg():
    return load_oracle()


def test_goldens_present():
    assert len(GOLDEN) >= 4


@pytest.mark.parametrize("path", GOLDEN, ids=lambda p: p.stem)
def test_capture_field_matches_reference(cg, path):
    z = np.load(path)
    p, e, _ = grids(z)
    fp = z["footprints"]
    field = cg.capture_field(p["states"], e["states"], fp[:2], fp[2:],
                             float(z["exit_radius"]))
    np.testing.assert_allclose(field, z["frames"][0], rtol=0, atol=1e-12)


@pytest.mark.parametrize("path", GOLDEN, ids=lambda p: p.stem)
def test_dense_backup_matches_joint_enumeration(cg, path):
    z = np.load(path)
    p, e, _ = grids(z)
    frames = z["frames"]
    for k in range(len(frames) - 1):
        out = cg.backup_dense(frames[k], p, e, float(z["exit_radius"]))
        np.testing.assert_allclose(out, frames[k + 1], rtol=0, atol=1e-12)


@pytest.mark.parametrize("path", GOLDEN, ids=lambda p: p.stem)
def test_packed_backup_preserves_the_game(cg, path):
    z = np.load(path)
    p, e, domain = grids(z)
    frames = z["frames"]
    n_p, n_e = frames.shape[1:]
    radius = domain["exit_radius"]
    flat = cg.pack(frames[0], domain)
    np.testing.assert_array_equal(cg.expand_packed(flat, domain, n_p, n_e, radius),
                                  np.where(frames[0] == radius, radius, frames[0]))
    for k in range(len(frames) - 1):
        flat = cg.backup_packed(flat, p, e, domain)
        np.testing.assert_allclose(cg.expand_packed(flat, domain, n_p, n_e, radius),
                                   frames[k + 1], rtol=0, atol=1e-12)


def test_packed_query_reads_the_product_stencil(cg):
    z = np.load(GOLDEN[0])
    p, e, domain = grids(z)
    frames = z["frames"]
    n_p, n_e = frames.shape[1:]
    flat = cg.pack(frames[1], domain)
    rng = np.random.default_rng(3)
    n = 12
    pi = rng.integers(n_p, size=(n, 16)).astype(np.int32)
    ei = rng.integers(n_e, size=(n, 16)).astype(np.int32)
    pw = rng.random((n, 16)) * (rng.random((n, 16)) > 0.3)
    ew = rng.random((n, 16)) * (rng.random((n, 16)) > 0.3)
    dense = cg.expand_packed(flat, domain, n_p, n_e, domain["exit_radius"])
    expected = np.einsum("na,nb,nab->n", pw, ew, dense[pi[:, :, None], ei[:, None, :]])
    np.testing.assert_allclose(
        cg.query_packed(flat, pi, pw, ei, ew, domain, n_e), expected, atol=1e-12)


def test_arena_clearance_equals_the_reference_values():
    """Signed rectangle clearance from walls and circles on the host, against
    the reference CircleArena.clearance at golden random states."""
    from pathlib import Path

    from pursuit_evasion_b200.local_game.geometry import CircleArena

    z = np.load(Path(__file__).resolve().parent / "golden" / "vehicle_grid_posts3m.npz")
    arena = CircleArena(z["circles"], float(z["half_width"]))
    np.testing.assert_allclose(arena.clearance(z["query_states"], "evader"),
                               z["query_clearance"], rtol=0, atol=1e-12)
