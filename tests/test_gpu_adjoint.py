"""Gradients of eigenray TL and travel time (underseamodelinglibrary_b200
.adjoint) against central differences of the CPU oracle (the FP64
restatement of the reference): the engine's reverse sweep for the
sound-speed nodes, the exact bottom-parameter derivatives of the
sensitivity mode, and the torch.autograd.Function wrapper.

Tolerance: 1e-3 of the difference quotient, as the differentiation
contract states, plus an absolute floor of 1e-6 dB or 1e-9 s per m/s for
derivatives the difference step cannot resolve."""
import numpy as np
import pytest

from underseamodelinglibrary_b200 import adjoint as A
from oracle_binding import OracleQueue

pytestmark = pytest.mark.gpu

REL = 1e-3


def small():
    return A.AdjointScenario(num_de=181, num_az=19, n_steps=240, n_targets=12, max_range=15e3)


def oracle_rays(sc, nodes, bottom=None):
    ocean = sc.ocean(nodes, bottom)
    q = OracleQueue(ocean, sc.freq, sc.pos, sc.de, sc.az, sc.dt, sc.targets)
    q.run(sc.time_max)
    return {A._key(r): r for r in q.take_eigenrays()}


@pytest.fixture(scope="module")
def prop():
    sc = small()
    nodes = A.munk_nodes()
    return sc, nodes, A.Propagation(sc, nodes, checkpoint=50)


@pytest.fixture(scope="module")
def oracle_fd(prop):
    """central differences of the oracle, step 1e-3 c_k, for every node"""
    sc, nodes, _ = prop
    out = []
    for k in range(nodes.size):
        h = 1e-3 * abs(nodes[k])
        cp, cm = nodes.copy(), nodes.copy()
        cp[k] += h
        cm[k] -= h
        out.append((h, oracle_rays(sc, cp), oracle_rays(sc, cm)))
    return out


def test_bottom_derivatives_match_oracle_differences(prop):
    sc, nodes, p = prop
    rays = p.eigenrays
    assert len(rays) > 20
    assert any(r.bottom > 0 for r in rays)
    for j in range(3):
        # near the critical angle the loss bends sharply, so the oracle's
        # difference needs a small step to reach the derivative
        h = 1e-6 * sc.bottom[j]
        bp, bm = list(sc.bottom), list(sc.bottom)
        bp[j] += h
        bm[j] -= h
        plus, minus = oracle_rays(sc, nodes, tuple(bp)), oracle_rays(sc, nodes, tuple(bm))
        checked = 0
        for i, r in enumerate(rays):
            k = A._key(r)
            if k not in plus or k not in minus:
                continue
            fd = (plus[k].intensity[0] - minus[k].intensity[0]) / (2 * h)
            an = p.d_bottom[i, j]
            assert abs(an - fd) <= REL * max(abs(fd), 1e-6), (k, j, an, fd)
            checked += 1
        assert checked > 20


def test_adjoint_rows_match_oracle_differences(prop, oracle_fd):
    """Jacobian rows from unit-weight reverse sweeps against the oracle's
    central differences, node by node, on eigenrays whose (step, target,
    D/E, AZ) bracket holds under both perturbations."""
    sc, nodes, p = prop
    rays = p.eigenrays
    rng = np.random.default_rng(7)
    idx = sorted(rng.choice(len(rays), size=min(12, len(rays)), replace=False))
    rows = p.rows(idx)
    checked = 0
    for r_i, i in enumerate(idx):
        key = A._key(rays[i])
        for k, (h, plus, minus) in enumerate(oracle_fd):
            if key not in plus or key not in minus:
                continue
            fd_tl = (plus[key].intensity[0] - minus[key].intensity[0]) / (2 * h)
            fd_t = (plus[key].travel_time - minus[key].travel_time) / (2 * h)
            assert abs(rows[r_i, 0, k] - fd_tl) <= REL * abs(fd_tl) + 1e-6, (key, k, rows[r_i, 0, k], fd_tl)
            assert abs(rows[r_i, 1, k] - fd_t) <= REL * abs(fd_t) + 1e-9, (key, k, rows[r_i, 1, k], fd_t)
            checked += 1
    assert checked > 100


def test_vjp_matches_weighted_oracle_differences(prop, oracle_fd):
    """one reverse sweep with weights on every eigenray equals the same
    weighted sum of the oracle's differences (eigenrays whose topology
    changes under a perturbation carry no weight)"""
    sc, nodes, p = prop
    rays = p.eigenrays
    keys = [A._key(r) for r in rays]
    stable = np.array([all(k in plus and k in minus for _, plus, minus in oracle_fd) for k in keys])
    assert stable.sum() > 0.5 * len(rays)
    rng = np.random.default_rng(11)
    w_tl = rng.normal(size=len(rays)) * stable
    w_t = rng.normal(size=len(rays)) * stable * 1000.0
    g, gb, ms = p.vjp(w_tl, w_t)
    assert ms > 0.0
    for k, (h, plus, minus) in enumerate(oracle_fd):
        fd = 0.0
        for i, key in enumerate(keys):
            if stable[i]:
                fd += w_tl[i] * (plus[key].intensity[0] - minus[key].intensity[0]) / (2 * h)
                fd += w_t[i] * (plus[key].travel_time - minus[key].travel_time) / (2 * h)
        assert abs(g[k] - fd) <= REL * abs(fd) + 1e-5, (k, g[k], fd)
    assert np.allclose(gb, w_tl @ p.d_bottom, rtol=1e-12, atol=0)


def test_torch_function_backward(engine):
    torch = pytest.importorskip("torch")
    sc = A.AdjointScenario(num_de=91, num_az=13, n_steps=160, n_targets=6, max_range=10e3)
    nodes = torch.tensor(A.munk_nodes(), dtype=torch.float64, requires_grad=True)
    bottom = torch.tensor(sc.bottom, dtype=torch.float64, requires_grad=True)
    f = A.EigenrayTLTime
    vals = f.apply(nodes, bottom, sc)
    assert vals.shape[1] == 2 and vals.shape[0] > 3
    w = torch.linspace(0.5, 1.5, vals.shape[0], dtype=torch.float64)
    (vals[:, 0] * w + 100.0 * vals[:, 1]).sum().backward()
    p = A.Propagation(sc, nodes.detach().numpy())
    g, gb, _ = p.vjp(w.numpy(), np.full(vals.shape[0], 100.0))
    assert np.allclose(nodes.grad.numpy(), g, rtol=1e-9, atol=1e-12)
    assert np.allclose(bottom.grad.numpy(), gb, rtol=1e-9, atol=1e-12)
