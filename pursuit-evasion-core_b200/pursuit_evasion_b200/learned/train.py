"""Training and inference drivers of the value surrogate on solver tables.

`NodeSampler` turns flat grid-node indices of a device-resident table into
(feature, value) minibatches with the encode kernels of csrc/mlp.cu;
`train` runs Adam on a fixed set of sampled pairs (epochs over a permuted
index list, one CUDA graph replay per step); `predict_nodes` evaluates the
surrogate on every node of a grid (the warm start of value iteration);
`predict_states` answers online queries of arbitrary relative states.
"""

from __future__ import annotations

import ctypes
import time

import numpy as np

from .. import _native
from .mlp import FEATURES, ValueMLP, _ptr


class RelativeNodeSampler:
    """Relative 5D grid nodes [vP, vE, psi, y, x] of a dense table."""

    in_features = 6

    def __init__(self, config, grid, table=None):
        self.grid = grid
        self.table = table  # torch float32 tensor (dense) or None for inference
        p, e = config.pursuer, config.evader
        self.args = (grid.positions, grid.headings, grid.p_speeds, grid.e_speeds,
                     float(grid.extent), float(p.speed_min), float(p.speed_max),
                     float(e.speed_min), float(e.speed_max))
        self.cells = grid.states

    def encode(self, net, idx, rows, with_target):
        lib = _native.library()
        _native.check(lib.pe_mlp_encode_relative_nodes(
            _ptr(self.table) if with_target else None, _ptr(idx), rows, *self.args,
            _ptr(net.feat), FEATURES, _ptr(net.target) if with_target else None,
            net._stream()))


class WorldNodeSampler:
    """8D grid nodes [xP, yP, thP, vP, xE, yE, thE, vE] of a dense table."""

    in_features = 10

    def __init__(self, config, grid, table=None):
        self.grid = grid
        self.table = table
        p, e = config.pursuer, config.evader
        self.args = (grid.positions, grid.headings, grid.p_speeds, grid.e_speeds,
                     float(grid.extent), float(p.speed_min), float(p.speed_max),
                     float(e.speed_min), float(e.speed_max))
        self.cells = grid.states

    def encode(self, net, idx, rows, with_target):
        lib = _native.library()
        _native.check(lib.pe_mlp_encode_world_nodes(
            _ptr(self.table) if with_target else None, _ptr(idx), rows, *self.args,
            _ptr(net.feat), FEATURES, _ptr(net.target) if with_target else None,
            net._stream()))


def train(net, sampler, *, samples=1 << 22, epochs=20, batch=8192, lr=1e-3,
          seed=0, use_graph=True, log=None):
    """Adam on `samples` node pairs drawn uniformly (with replacement) from
    the sampler's table; returns per-epoch mean losses and the wall time."""
    torch = net.torch
    if batch > net.batch:
        raise ValueError("batch exceeds the network's buffers")
    dev = net.dev
    gen = torch.Generator(device=dev).manual_seed(seed)
    dataset = torch.randint(sampler.cells, (samples,), generator=gen, device=dev)
    steps_per_epoch = samples // batch
    idx = torch.empty(batch, dtype=torch.int64, device=dev)

    def step_body():
        net.loss.zero_()
        sampler.encode(net, idx, batch, True)
        net.forward(batch, target=True)
        net.backward(batch)
        net.adam(lr=lr)

    stream = torch.cuda.Stream(device=dev)
    graph = None
    losses = []
    started = time.perf_counter()
    step = 0
    with torch.cuda.stream(stream):
        for epoch in range(epochs):
            order = torch.randperm(samples, generator=gen, device=dev)
            epoch_loss = torch.zeros(1, device=dev)
            for k in range(steps_per_epoch):
                step += 1
                idx.copy_(dataset[order[k * batch:(k + 1) * batch]])
                net.set_step(step)
                if use_graph and graph is None and step >= 3:
                    torch.cuda.synchronize(dev)
                    graph = torch.cuda.CUDAGraph()
                    with torch.cuda.graph(graph, stream=stream):
                        step_body()
                if graph is not None:
                    graph.replay()
                else:
                    step_body()
                epoch_loss += net.loss
            losses.append(float(epoch_loss) / steps_per_epoch)
            if log:
                log(f"epoch {epoch + 1}: mse {losses[-1]:.3e}")
    torch.cuda.synchronize(dev)
    return losses, time.perf_counter() - started


def predict_nodes(net, sampler, out, *, chunk=8192):
    """Surrogate value at every grid node into the float32 device tensor `out`."""
    torch = net.torch
    dev = net.dev
    n = sampler.cells
    chunk = min(chunk, net.batch)
    idx = torch.empty(chunk, dtype=torch.int64, device=dev)
    for start in range(0, n, chunk):
        rows = min(chunk, n - start)
        padded = (rows + 127) // 128 * 128
        torch.arange(start, start + padded, out=idx[:padded], device=dev)
        idx[:padded].clamp_(max=n - 1)
        sampler.encode(net, idx, padded, False)
        y = net.forward(padded, inference=True)
        out[start:start + rows].copy_(y[:rows])
    return out


def predict_states(net, config, extent, states):
    """Online query: surrogate values of relative states [n][5] (device)."""
    torch = net.torch
    n = states.shape[0]
    padded = (n + 127) // 128 * 128
    if padded > net.batch:
        raise ValueError("query batch exceeds the network's buffers")
    p, e = config.pursuer, config.evader
    lib = _native.library()
    _native.check(lib.pe_mlp_encode_relative_states(
        _ptr(states), n, float(extent), float(p.speed_min), float(p.speed_max),
        float(e.speed_min), float(e.speed_max), _ptr(net.feat), FEATURES, net._stream()))
    if padded > n:
        net.feat[n:padded].zero_()
    # the network's output buffer is reused: copy the answers out
    return net.forward(padded, inference=True)[:n].clone()
