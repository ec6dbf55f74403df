"""CPU ORACLE -- test infrastructure only.

Only tests/, the smoke check and bench.py's CPU-baseline leg may import this
module, and only as the checker.  It is never the product path.

FP64 NumPy restatement of the reference's compact eight-state
semi-Lagrangian contact game (pursuit-evasion-core
src/pursuit_evasion/local_game/grid_game.py):

  * capture field: oriented-rectangle separating-axis value of the two
    footprints, `exit_radius` where the centres are farther apart
    (grid_game.py:193-201 `initialize`, geometry.py:15-36);
  * one backup: for every cell (ip, ie) within the exit radius,
        out = min(V, min_{u allowed at ip} max_{a allowed at ie}
                  sum_q we[ie,a,q] sum_k wp[ip,u,k] V[idp[ip,u,k], ide[ie,a,q]])
    the factorized product interpolation of grid_game.py:202-221
    (`interpolate_p` then `reduce_e`, with `backup_gpu`'s chunk/action
    loop :286-333 folding the running minimum through the P actions).  The
    reference's early exit (`worst >= best`) only skips P actions that
    cannot lower the minimum, so the value equals this plain min-max;
  * the pair-packed domain (grid_game.py:336-381 `PairDomain`,
    :384-421 `p_packed` / `e_packed`): only pairs within the exit radius are
    stored; an interpolation vertex outside the domain, or an evader state
    beyond `reach` of the pursuer, reads `exit_value`;
  * the packed query (reference.py:122-134 `query_field`).

Pinned against golden vectors that the reference's own test helpers
produced (tests/golden/make_compact_golden.py: `fake_grid`,
`brute_backup`, tests/test_compact_dp.py:12-51).
"""

from __future__ import annotations

import numpy as np


def rectangle_separation(p, e, p_body, e_body):
    """geometry.py:15-36: max of the four separating-axis gaps (FP64)."""
    p, e = np.asarray(p, np.float64), np.asarray(e, np.float64)
    d = e[..., :2] - p[..., :2]
    delta = e[..., 2] - p[..., 2]
    ca, sa = np.abs(np.cos(delta)), np.abs(np.sin(delta))
    values = []
    for pose, own, other in ((p, p_body, e_body), (e, e_body, p_body)):
        c, s = np.cos(pose[..., 2]), np.sin(pose[..., 2])
        x = d[..., 0] * c + d[..., 1] * s
        y = -d[..., 0] * s + d[..., 1] * c
        values.append(np.abs(x) - own[0] / 2 - (other[0] * ca + other[1] * sa) / 2)
        values.append(np.abs(y) - own[1] / 2 - (other[0] * sa + other[1] * ca) / 2)
    return np.maximum.reduce(values)


def capture_field(p_states, e_states, p_body, e_body, exit_radius):
    """Dense [np, ne] initial field (grid_game.py:193-201)."""
    field = rectangle_separation(p_states[:, None], e_states[None], p_body, e_body)
    dist2 = ((p_states[:, None, :2] - e_states[None, :, :2]) ** 2).sum(-1)
    return np.where(dist2 > exit_radius ** 2, exit_radius, field)


def _interpolate_p(f, ids, w, allowed, ip, u):
    """Row g[ie'] = sum_k w[ip,u,k] f[ids[ip,u,k], ie'] (zero weights skipped)."""
    if not allowed[ip, u]:
        return np.zeros(f.shape[1])
    k = w[ip, u] > 0
    return (w[ip, u, k, None] * f[ids[ip, u, k]]).sum(0)


def backup_dense(f, p, e, exit_radius):
    """One backup of the dense [np, ne] field; p and e carry states,
    successors [n, na, 16], weights [n, na, 16] and allowed [n, na]."""
    f = np.asarray(f, np.float64)
    out = f.copy()
    n_p, n_e = f.shape
    near = ((p["states"][:, None, :2] - e["states"][None, :, :2]) ** 2).sum(-1) <= exit_radius ** 2
    ew = e["weights"].astype(np.float64)
    eid = e["successors"]
    for ip in range(n_p):
        cells = np.flatnonzero(near[ip])
        if not len(cells):
            continue
        best = out[ip, cells].copy()
        for u in np.flatnonzero(p["allowed"][ip]):
            g = _interpolate_p(f, p["successors"], p["weights"].astype(np.float64),
                               p["allowed"], ip, u)
            # value[cell, a] = sum_q we[ie,a,q] g[ide[ie,a,q]]
            value = (np.where(ew[cells] > 0, ew[cells], 0) * g[eid[cells]]).sum(-1)
            value = np.where(e["allowed"][cells], value, -1e30)
            worst = value.max(-1)
            best = np.minimum(best, worst)
        out[ip, cells] = best
    return out


def expand_packed(flat, domain, n_p, n_e, exit_value):
    """Packed pair vector -> dense [np, ne] (exit_value outside the domain)."""
    out = np.full((n_p, n_e), exit_value, np.float64)
    for i in range(n_p):
        pos = domain["p_position"][i]
        ids = domain["e_indices"][pos, : domain["counts"][pos]]
        out[i, ids] = flat[domain["offsets"][i]: domain["offsets"][i + 1]]
    return out


def pack(dense, domain):
    """Dense [np, ne] -> packed pair vector."""
    parts = []
    for i in range(dense.shape[0]):
        pos = domain["p_position"][i]
        parts.append(dense[i, domain["e_indices"][pos, : domain["counts"][pos]]])
    return np.concatenate(parts)


def e_reach(e):
    """Largest centre displacement of an evader interpolation vertex with a
    positive weight, plus 1e-4 (grid_game.py:456-466)."""
    ids, w, s = e["successors"], e["weights"], e["states"]
    dist = np.linalg.norm(s[ids, :2] - s[:, None, None, :2], axis=-1)
    return float(np.where(w > 0, dist, 0).max()) + 1e-4


def backup_packed(flat, p, e, domain, ips=None):
    """One backup of the packed pair vector (grid_game.py:384-421); with
    `ips`, only the pairs of those pursuer states are updated."""
    radius = float(domain["exit_radius"])
    n_p, n_e = len(p["states"]), len(e["states"])
    reach = radius + e_reach(e)
    out = np.asarray(flat, np.float64).copy()
    lookup, offsets, ppos = domain["lookup"], domain["offsets"], domain["p_position"]
    ew = e["weights"].astype(np.float64)
    eid = e["successors"]
    for ip in range(n_p) if ips is None else ips:
        pos = ppos[ip]
        cells_e = domain["e_indices"][pos, : domain["counts"][pos]]
        if not len(cells_e):
            continue
        dest = offsets[ip] + np.arange(len(cells_e))
        best = out[dest].copy()
        far = ((p["states"][ip, :2] - e["states"][:, :2]) ** 2).sum(-1) > reach ** 2
        for u in np.flatnonzero(p["allowed"][ip]):
            g = np.zeros(n_e)
            for k in range(16):
                wk = float(p["weights"][ip, u, k])
                if wk <= 0:
                    continue
                nxt = p["successors"][ip, u, k]
                rank = lookup[ppos[nxt]]
                vals = np.where(rank < 0, radius,
                                flat[np.clip(offsets[nxt] + rank, 0, len(flat) - 1)])
                g += wk * vals
            g = np.where(far, radius, g)
            value = (np.where(ew[cells_e] > 0, ew[cells_e], 0) * g[eid[cells_e]]).sum(-1)
            value = np.where(e["allowed"][cells_e], value, -1e30)
            best = np.minimum(best, value.max(-1))
        out[dest] = best
    return out


def query_packed(flat, pi, pw, ei, ew, domain, n_e):
    """reference.py:122-134: product-stencil query of the packed field."""
    radius = float(domain["exit_radius"])
    out = np.zeros(len(pi))
    for i in range(len(pi)):
        total = 0.0
        for a in range(16):
            if pw[i, a] <= 0:
                continue
            value = 0.0
            for b in range(16):
                if ew[i, b] <= 0:
                    continue
                rank = domain["lookup"][domain["p_position"][pi[i, a]], ei[i, b]]
                value += ew[i, b] * (radius if rank < 0
                                     else flat[domain["offsets"][pi[i, a]] + rank])
            total += pw[i, a] * value
        out[i] = total
    return out
