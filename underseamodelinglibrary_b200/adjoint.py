"""Gradients of eigenray transmission loss and travel time at receivers
with respect to a piecewise-linear sound-speed profile (profile_grid<1>
nodes) and the Rayleigh bottom parameters, at the forward pass's frozen
eigenray topology.

* d TL / d c_j and d T / d c_j (profile nodes): the engine's reverse sweep
  (wq3d_queue_enable_adjoint / wq3d_queue_adjoint).  The forward pass keeps
  every ray's state every K steps and each eigenray's partial derivatives
  with respect to the fronts it was built from; the sweep recomputes each
  checkpoint interval and runs the adjoint of the AB3 steps, the reflection
  chains and the start-up back through it.  One sweep gives one weighted
  sum of the rows (a vector-Jacobian product); a row of the Jacobian is a
  sweep with one unit weight.
* d TL / d bottom (density ratio, speed ratio, attenuation in dB per
  wavelength): exact, from the GPU's sensitivity mode
  (wq3d_queue_enable_sensitivity).  The reflection loss does not move the
  rays, so each ray's accumulated loss derivative is the whole derivative;
  travel time does not depend on these parameters.
* ``finite_differences`` keeps the batched central differences of the FP64
  GPU form (2 x nodes perturbed propagations run together), the check the
  adjoint is held to.

``EigenrayTLTime`` is a torch.autograd.Function over these: forward gives
(TL at the first frequency, travel time) per eigenray, backward is one
reverse sweep.
"""
import math

import numpy as np

from . import _abi
from . import types as T
from .ocean import (attenuation_thorp, boundary_flat, data_grid, ocean_model, profile_grid,
                    reflect_loss_rayleigh)
from .waveq3d import run_batch, wave_queue


def munk_nodes(n_nodes=20, seed=20261203, std=2.0, depth=5000.0):
    """Munk sound speed at n_nodes equally spaced depths 0..depth, plus
    seeded N(0, std^2) perturbations: the parameter vector of the
    differentiable workload."""
    z = np.linspace(0.0, depth, n_nodes)
    zt = 2.0 * (z - 1300.0) / 1300.0
    c = 1500.0 * (1.0 + 0.00737 * (zt - 1.0 + np.exp(-zt)))
    return c + np.random.default_rng(seed).normal(0.0, std, n_nodes)


class AdjointScenario:
    """Flat 5000 m bottom with a Rayleigh loss, a 20-node profile_grid<1>
    (linear in depth, rho axis descending), Thorp absorption, source at 45N
    45W 1000 m deep, receivers at random range 1-50 km, bearing and depth
    10-4900 m.  Defaults are the full workload: 1801 x 91 rays, dt 0.05 s,
    2000 steps, 64 receivers, 1 kHz."""

    def __init__(self, num_de=1801, num_az=91, n_steps=2000, n_targets=64, dt=0.05, freq=1000.0,
                 bottom=(1.8, 1.15, 0.3), seed=20261203, depth=5000.0, max_range=50e3):
        T.compute_earth_radius(45.0)
        self.earth_radius = T.earth_radius()
        self.num_de, self.num_az = num_de, num_az
        self.dt = dt
        self.n_steps = n_steps
        self.time_max = (n_steps - 0.5) * dt
        self.freq = T.seq_log(freq, 1.0, 1)
        self.depth = depth
        self.bottom = tuple(float(x) for x in bottom)
        self.pos = T.wposition1(45.0, -45.0, -1000.0)
        rng = np.random.default_rng(seed + 1)
        self.targets = T.wposition(1, n_targets, 0.0, 0.0, 0.0)
        for j in range(n_targets):
            p = T.wposition1(self.pos, float(rng.uniform(1e3, max_range)), float(rng.uniform(0.0, 2 * math.pi)))
            self.targets.latitude(0, j, p.latitude())
            self.targets.longitude(0, j, p.longitude())
            self.targets.altitude(0, j, -float(rng.uniform(10.0, depth - 100.0)))
        self.de = T.seq_rayfan(-90.0, 90.0, num_de)
        self.az = T.seq_linear(0.0, 360.0 / (num_az - 1), num_az)

    def ocean(self, nodes, bottom=None):
        T.set_earth_radius(self.earth_radius)
        nodes = np.asarray(nodes, dtype=np.float64)
        R = self.earth_radius
        ax = T.seq_linear(R, -self.depth / (nodes.size - 1), nodes.size)
        g = data_grid([ax], nodes)
        b = self.bottom if bottom is None else bottom
        return ocean_model(boundary_flat(), boundary_flat(self.depth, reflect_loss_rayleigh(*b)),
                           profile_grid(g, attenuation_thorp()))

    def queue(self, nodes, bottom=None, precision=_abi.FP64):
        T.set_earth_radius(self.earth_radius)
        return wave_queue(self.ocean(nodes, bottom), self.freq, self.pos, self.de, self.az, self.dt,
                          self.targets, precision=precision)


def _key(r):
    return (r.step, r.t1, r.t2, r.de_index, r.az_index)


class Propagation:
    """One forward pass recorded for the reverse sweep: ``eigenrays``,
    ``values`` (n x 2: TL of the first frequency, travel time),
    ``d_bottom`` (n x 3, exact TL derivatives with respect to the bottom
    parameters) and ``ms_forward`` (device ms).  ``vjp`` and ``rows`` run
    reverse sweeps on it."""

    def __init__(self, sc, nodes, checkpoint=50, precision=_abi.FP64, max_eigenrays=0):
        self.nodes = np.asarray(nodes, dtype=np.float64)
        q = sc.queue(self.nodes, precision=precision)
        q.enable_sensitivity()
        q.enable_adjoint(checkpoint, sc.n_steps + 16, max_eigenrays)
        q.timing(reset=True)
        q.run(sc.time_max)
        self.ms_forward = q.timing()["total_ms"]
        self.queue = q
        self.eigenrays = q.take_eigenrays()
        cols = self.eigenrays.arrays()
        n = len(self.eigenrays)
        self.values = np.stack([cols["intensity"][:, 0], cols["time"]], axis=1) if n else np.zeros((0, 2))
        self.d_bottom = cols.get("d_intensity_d_bottom", np.zeros((n, 3)))

    def vjp(self, w_tl, w_time):
        """(d/d nodes, d/d bottom, device ms) of sum_k w_tl[k] TL_k +
        w_time[k] T_k: one reverse sweep."""
        w_tl = np.asarray(w_tl, dtype=np.float64)
        w_time = np.asarray(w_time, dtype=np.float64)
        g, ms = self.queue.adjoint(self.eigenrays, w_tl, w_time, self.nodes.size)
        gb = w_tl @ self.d_bottom if len(w_tl) else np.zeros(3)
        return g, gb, ms

    def rows(self, indices):
        """Jacobian rows (len(indices) x 2 x (nodes + 3)) of the chosen
        eigenrays: two unit-weight sweeps per eigenray."""
        n = len(self.eigenrays)
        out = np.zeros((len(indices), 2, self.nodes.size + 3))
        for r, i in enumerate(indices):
            w = np.zeros(n)
            w[i] = 1.0
            out[r, 0, :self.nodes.size], _ = self.queue.adjoint(self.eigenrays, w, np.zeros(n), self.nodes.size)
            out[r, 1, :self.nodes.size], _ = self.queue.adjoint(self.eigenrays, np.zeros(n), w, self.nodes.size)
            out[r, 0, self.nodes.size:] = self.d_bottom[i]
        return out


def finite_differences(sc, nodes, rel_step=1e-3):
    """Central differences of the FP64 GPU form for every eigenray and
    node: (eigenrays, jacobian n x 2 x nodes, device ms).  An eigenray whose
    (step, target, D/E, AZ) bracket is not found in both perturbed runs
    gets NaN."""
    nodes = np.asarray(nodes, dtype=np.float64)
    q = sc.queue(nodes)
    q.run(sc.time_max)
    rays = q.take_eigenrays()
    nk = nodes.size
    qs, hs = [], []
    for k in range(nk):
        h = rel_step * abs(nodes[k])
        hs.append(h)
        for sgn in (1.0, -1.0):
            c = nodes.copy()
            c[k] += sgn * h
            qs.append(sc.queue(c))
    _, ms = run_batch(qs, sc.time_max)
    jac = np.full((len(rays), 2, nk), np.nan)
    index = {_key(r): i for i, r in enumerate(rays)}
    for k in range(nk):
        plus = {_key(r): r for r in qs[2 * k].take_eigenrays()}
        minus = {_key(r): r for r in qs[2 * k + 1].take_eigenrays()}
        for kk, i in index.items():
            if kk in plus and kk in minus:
                jac[i, 0, k] = (plus[kk].intensity[0] - minus[kk].intensity[0]) / (2 * hs[k])
                jac[i, 1, k] = (plus[kk].travel_time - minus[kk].travel_time) / (2 * hs[k])
    return rays, jac, ms


def _torch_function():
    import torch

    class EigenrayTLTime(torch.autograd.Function):
        """forward(nodes[k], bottom[3], scenario) -> (n, 2) tensor of
        (TL, travel time) per eigenray; backward is one reverse sweep of the
        engine's adjoint (and the exact bottom sensitivities)."""

        @staticmethod
        def forward(ctx, nodes, bottom, sc):
            b = tuple(float(x) for x in bottom.detach().cpu().numpy())
            if b != sc.bottom:
                sc.bottom = b
            prop = Propagation(sc, nodes.detach().cpu().numpy())
            ctx.prop = prop
            ctx.dtype = nodes.dtype
            return torch.as_tensor(prop.values, dtype=nodes.dtype)

        @staticmethod
        def backward(ctx, grad_out):
            g = grad_out.detach().cpu().numpy().astype(np.float64)
            gn, gb, _ = ctx.prop.vjp(g[:, 0], g[:, 1])
            return torch.as_tensor(gn, dtype=ctx.dtype), torch.as_tensor(gb, dtype=ctx.dtype), None

    return EigenrayTLTime


def __getattr__(name):
    if name == "EigenrayTLTime":
        return _torch_function()
    raise AttributeError(name)
