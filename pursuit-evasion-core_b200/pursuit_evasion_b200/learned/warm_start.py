"""Learned warm start of minimum-time value iteration, and its evaluation.

The plain DP decides the answer: `time_to_converged` solves the
relative 5D minimum-time game (semi-Lagrangian value iteration, a
contraction) to a sup-norm residual `tol` from the cold start (u = 1 outside
the capture disk) and again from a surrogate prediction, and reports the
iterations, device seconds and the largest difference between the two
converged tables.  The surrogate is trained by this package's kernels on
node samples of a solver table: the same problem's table (an amortised
re-solve) or a coarser grid's table (a multigrid-style cold path, whose cost
includes that coarse solve and the training).
"""

from __future__ import annotations

import time

from ..reversible.free_dp import RelativeGrid
from ..reversible.semilag import SemiLagrangianSolver
from .mlp import ValueMLP
from .train import RelativeNodeSampler, predict_nodes, train


INFER_CHUNK = 1 << 17  # rows per inference launch sequence


def converge(config, grid, *, dt, tol, initial=None, max_iterations=20000,
             check_every=5, device=0):
    """Minimum-time value iteration to residual < tol.  `initial`: optional
    dense float32 torch tensor on the device.  Returns (u tensor, info)."""
    import torch

    dev = torch.device("cuda", device)
    u = torch.empty(grid.states, device=dev)
    # the handle and the timing events share one explicit stream, ordered
    # after the work that produced `initial`
    stream = torch.cuda.Stream(device=dev)
    stream.wait_stream(torch.cuda.current_stream(dev))
    with SemiLagrangianSolver(config, grid, dt=dt, mode="min_time", device=device) as s, \
            torch.cuda.stream(stream):
        s.set_stream(stream.cuda_stream)
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if initial is not None:
            s.initialize_device(initial.data_ptr())
        else:
            s.initialize()
        start.record(stream)
        iters, residual, converged = s.iterate(max_iterations, tol=tol,
                                               check_every=check_every)
        end.record(stream)
        s.value_to_device(u.data_ptr())
        torch.cuda.synchronize(dev)
        seconds = start.elapsed_time(end) / 1e3
        computed = s.items_computed()
        items = s.tile["items"] if s.kernel == "tiled" else 0
    info = dict(iterations=iters, residual=residual, converged=converged, seconds=seconds)
    if items:
        # work skipping: the share of tiled work items actually computed
        info["items_computed_fraction"] = computed / (items * max(iters, 1))
    return u, info


def surrogate_start(net, config, grid, out):
    """Surrogate prediction on every node of `grid`, clamped to [0, 1]."""
    import torch

    predict_nodes(net, RelativeNodeSampler(config, grid), out, chunk=net.batch)
    out.clamp_(0.0, 1.0)
    return out


def time_to_converged(config, grid, *, dt, tol=1e-5, samples=1 << 22, epochs=20,
                      batch=8192, coarse_grid=None, seed=0, device=0, log=None):
    import torch

    dev = torch.device("cuda", device)
    result = {"grid": grid.to_dict(), "dt": dt, "tol": tol, "samples": samples,
              "epochs": epochs, "batch": batch}
    u_plain, plain = converge(config, grid, dt=dt, tol=tol, device=device)
    result["plain"] = plain

    def warm_from(table_grid, table, label):
        net = ValueMLP(RelativeNodeSampler.in_features, seed=seed, device=device,
                       max_batch=batch)
        losses, train_s = train(net, RelativeNodeSampler(config, table_grid, table),
                                samples=samples, epochs=epochs, batch=batch, seed=seed,
                                log=log)
        net.set_batch(INFER_CHUNK)  # inference in large chunks
        t0 = time.perf_counter()
        u0 = surrogate_start(net, config, grid, torch.empty(grid.states, device=dev))
        torch.cuda.synchronize(dev)
        infer_s = time.perf_counter() - t0
        surrogate_err = float((u0 - u_plain).abs().max())
        surrogate_mean = float((u0 - u_plain).abs().mean())
        u_warm, warm = converge(config, grid, dt=dt, tol=tol, initial=u0, device=device)
        warm.update(train_seconds=train_s, final_mse=losses[-1], inference_seconds=infer_s,
                    surrogate_max_abs_error=surrogate_err,
                    surrogate_mean_abs_error=surrogate_mean,
                    max_abs_diff_vs_plain=float((u_warm - u_plain).abs().max()),
                    speedup_iterations=plain["iterations"] / max(warm["iterations"], 1),
                    speedup_seconds=plain["seconds"] / max(warm["seconds"], 1e-12))
        result[label] = warm
        return net

    net = warm_from(grid, u_plain, "warm_same_table")
    w = result["warm_same_table"]
    # training and inference are charged: the surrogate is trained on this
    # very table, so this path only pays off when the network is reused
    w["end_to_end_seconds"] = w["train_seconds"] + w["inference_seconds"] + w["seconds"]
    w["speedup_end_to_end"] = plain["seconds"] / w["end_to_end_seconds"]
    if coarse_grid is not None:
        u_coarse, coarse = converge(config, coarse_grid, dt=dt, tol=tol, device=device)
        warm_from(coarse_grid, u_coarse, "warm_coarse_table")
        result["warm_coarse_table"]["coarse_solve"] = coarse
        w = result["warm_coarse_table"]
        w["end_to_end_seconds"] = (coarse["seconds"] + w["train_seconds"]
                                   + w["inference_seconds"] + w["seconds"])
        w["speedup_end_to_end"] = plain["seconds"] / w["end_to_end_seconds"]
    return result, net
