"""Gradients of eigenray transmission loss and travel time at receivers
with respect to a piecewise-linear sound-speed profile (profile_grid<1>
nodes) and the Rayleigh bottom parameters, at the forward pass's frozen
eigenray topology.

* d TL / d bottom (density ratio, speed ratio, attenuation in dB per
  wavelength): exact, from the GPU's sensitivity mode
  (wq3d_queue_enable_sensitivity).  The reflection loss does not move the
  rays, so the derivative of each ray's accumulated loss is the whole
  derivative; travel time does not depend on these parameters.
* d TL / d c_k and d T / d c_k: central differences of the FP64 GPU form
  with step h = rel_step * c_k, all 2 x nodes perturbed propagations run
  together by wq3d_batch_run.  An eigenray whose (step, target, D/E, AZ)
  bracket is not found in both perturbed runs gets NaN rows.  This is a
  numerical derivative of the discrete model, not an adjoint sweep.

``eigenray_gradients`` returns the Jacobian; ``EigenrayTLTime`` wraps it as
a torch.autograd.Function whose forward gives (TL at each frequency's
first entry, travel time) per eigenray and whose backward applies the
Jacobian's transpose.
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


def eigenray_gradients(sc, nodes, rel_step=1e-3, ssp=True):
    """Forward propagation plus gradients.  Returns a dict with
    ``eigenrays`` (eigenray_model list, reference order), ``values`` (n x 2:
    TL of the first frequency, travel time), ``jacobian`` (n x 2 x
    (nodes + 3)), ``ms_forward`` and ``ms_gradient`` (device ms)."""
    nodes = np.asarray(nodes, dtype=np.float64)
    nk = nodes.size
    q = sc.queue(nodes)
    q.enable_sensitivity()
    q.timing(reset=True)
    q.run(sc.time_max)
    ms_fwd = q.timing()["total_ms"]
    rays = q.take_eigenrays()
    n = len(rays)
    values = np.array([[r.intensity[0], r.travel_time] for r in rays]).reshape(n, 2)
    jac = np.zeros((n, 2, nk + 3))
    for i, r in enumerate(rays):
        jac[i, 0, nk:] = r.d_intensity_d_bottom
    ms_grad = 0.0
    if ssp and n > 0:
        qs, hs = [], []
        for k in range(nk):
            h = rel_step * abs(nodes[k])
            hs.append(h)
            for sgn in (1.0, -1.0):
                c = nodes.copy()
                c[k] += sgn * h
                qs.append(sc.queue(c))
        _, ms_grad = run_batch(qs, sc.time_max)
        index = {_key(r): i for i, r in enumerate(rays)}
        for k in range(nk):
            plus = {_key(r): r for r in qs[2 * k].take_eigenrays()}
            minus = {_key(r): r for r in qs[2 * k + 1].take_eigenrays()}
            for kk, i in index.items():
                if kk in plus and kk in minus:
                    jac[i, 0, k] = (plus[kk].intensity[0] - minus[kk].intensity[0]) / (2 * hs[k])
                    jac[i, 1, k] = (plus[kk].travel_time - minus[kk].travel_time) / (2 * hs[k])
                else:
                    jac[i, :, k] = np.nan
    return {"eigenrays": rays, "values": values, "jacobian": jac, "ms_forward": ms_fwd,
            "ms_gradient": ms_grad}


def _torch_function():
    import torch

    class EigenrayTLTime(torch.autograd.Function):
        """forward(nodes[k], bottom[3], scenario) -> (n, 2) tensor of
        (TL, travel time) per eigenray; backward applies the Jacobian of
        eigenray_gradients (NaN rows, for eigenrays whose topology changes
        under the perturbation, contribute zero)."""

        @staticmethod
        def forward(ctx, nodes, bottom, sc):
            b = tuple(float(x) for x in bottom.detach().cpu().numpy())
            if b != sc.bottom:
                sc.bottom = b
            out = eigenray_gradients(sc, nodes.detach().cpu().numpy())
            ctx.save_for_backward(torch.as_tensor(np.nan_to_num(out["jacobian"]), dtype=nodes.dtype))
            ctx.nk = nodes.numel()
            return torch.as_tensor(out["values"], dtype=nodes.dtype)

        @staticmethod
        def backward(ctx, grad_out):
            (jac,) = ctx.saved_tensors
            g = torch.einsum("ij,ijk->k", grad_out.to(jac.dtype), jac)
            return g[:ctx.nk], g[ctx.nk:], None

    return EigenrayTLTime


def __getattr__(name):
    if name == "EigenrayTLTime":
        return _torch_function()
    raise AttributeError(name)
