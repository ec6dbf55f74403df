"""GPU table queries (pe_table_*) against the host reader of the same table
(the restatement of the reference's RelativeTable): capture times and
signed fields of random, boundary, captured, out-of-box and non-finite
states, and batches whose bisection depths differ."""

import numpy as np
import pytest

from pursuit_evasion_b200.reversible.free_dp import RelativeGrid, solve
from pursuit_evasion_b200.reversible.relative_table import DeviceRelativeTable, RelativeTable
from tests.helpers import A3

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def table(tmp_path_factory):
    out = tmp_path_factory.mktemp("tab") / "t"
    solve(A3, RelativeGrid(13, 12, 7, 7, 3.0), out, horizon=1.0, output_dt=0.1,
          local_precision="float64")
    return RelativeTable(out, A3)


def random_states(table, n, seed):
    rng = np.random.default_rng(seed)
    ax = table.axes  # storage order [vP, vE, psi, y, x]
    s = np.stack([rng.uniform(ax[4][0] - 0.2, ax[4][-1] + 0.2, n),
                  rng.uniform(ax[3][0] - 0.2, ax[3][-1] + 0.2, n),
                  rng.uniform(-4, 4, n),
                  rng.uniform(ax[0][0], ax[0][-1], n),
                  rng.uniform(ax[1][0], ax[1][-1], n)], 1)
    # exact grid nodes, captured states, the heading seam, non-finite entries
    s[:5, 0] = ax[4][:5]
    s[5:10, :2] = 0.1
    s[10:15, 2] = np.pi
    s[15, 0] = np.nan
    s[16, 3] = np.inf
    return s


def close(a, b):
    both_nan = np.isnan(a) & np.isnan(b)
    assert np.array_equal(np.isnan(a), np.isnan(b))
    np.testing.assert_allclose(a[~both_nan], b[~both_nan], rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("n, seed", [(4096, 0), (37, 1), (1, 2)])
def test_capture_times_match_host_reader(table, n, seed):
    states = random_states(table, max(n, 20), seed)[:n]
    with DeviceRelativeTable(table) as dev:
        close(dev.value(states), table.value(states))


def test_signed_field_matches_host_reader(table):
    states = random_states(table, 2000, 3)
    budgets = np.random.default_rng(4).uniform(-0.1, 1.1, len(states))
    budgets[:10] = table.times[:10]
    with DeviceRelativeTable(table) as dev:
        close(dev.field(states, budgets), table.field(states, budgets))
        close(dev.field(states, 0.55), table.field(states, 0.55))


def test_batch_semantics_of_the_bisection(table):
    """States already inside at t = 0 (interpolated field <= 0 but outside
    the exact capture disk) resolve as in a reference batch, alone and with
    states that bisect one step longer."""
    r = A3.capture_radius
    inside = np.array([[r + 0.02, 0.0, 0.3, 0.5, 0.25], [0.0, r + 0.03, -1.0, 1.0, 0.5]])
    others = random_states(table, 300, 5)
    for batch in (inside, np.concatenate([inside, others])):
        with DeviceRelativeTable(table) as dev:
            close(dev.value(batch), table.value(batch))
    assert np.all(np.isnan(table.value(np.full((3, 5), np.nan))))
