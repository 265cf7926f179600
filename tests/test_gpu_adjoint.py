"""Gradients of eigenray TL and travel time (underseamodelinglibrary_b200
.adjoint) against central differences of the CPU oracle (the FP64
restatement of the reference): exact bottom-parameter derivatives from the
GPU's sensitivity mode, batched-difference sound-speed derivatives, and
the torch.autograd.Function wrapper."""
import numpy as np
import pytest

from underseamodelinglibrary_b200 import adjoint as A
from oracle_binding import OracleQueue

pytestmark = pytest.mark.gpu


def small():
    return A.AdjointScenario(num_de=181, num_az=19, n_steps=240, n_targets=12, max_range=15e3)


def oracle_rays(sc, nodes, bottom=None):
    ocean = sc.ocean(nodes, bottom)
    q = OracleQueue(ocean, sc.freq, sc.pos, sc.de, sc.az, sc.dt, sc.targets)
    q.run(sc.time_max)
    return {A._key(r): r for r in q.take_eigenrays()}


def test_bottom_derivatives_match_oracle_differences(engine):
    sc = small()
    nodes = A.munk_nodes()
    out = A.eigenray_gradients(sc, nodes, ssp=False)
    rays = out["eigenrays"]
    assert len(rays) > 20
    bounced = [i for i, r in enumerate(rays) if r.bottom > 0]
    assert bounced
    for p in range(3):
        # near the critical angle the loss bends sharply, so the oracle's
        # difference needs a small step to reach the derivative
        h = 1e-6 * sc.bottom[p]
        bp, bm = list(sc.bottom), list(sc.bottom)
        bp[p] += h
        bm[p] -= h
        plus, minus = oracle_rays(sc, nodes, tuple(bp)), oracle_rays(sc, nodes, tuple(bm))
        checked = 0
        for i, r in enumerate(rays):
            k = A._key(r)
            if k not in plus or k not in minus:
                continue
            fd = (plus[k].intensity[0] - minus[k].intensity[0]) / (2 * h)
            an = out["jacobian"][i, 0, nodes.size + p]
            assert abs(an - fd) <= 1e-3 * max(abs(fd), 1e-6), (k, p, an, fd)
            checked += 1
        assert checked > 20


def test_sound_speed_derivatives_match_oracle_differences(engine):
    sc = small()
    nodes = A.munk_nodes()
    out = A.eigenray_gradients(sc, nodes)
    rays = out["eigenrays"]
    for k_node in (2, 4, 9):
        h = 1e-3 * abs(nodes[k_node])
        cp, cm = nodes.copy(), nodes.copy()
        cp[k_node] += h
        cm[k_node] -= h
        plus, minus = oracle_rays(sc, cp), oracle_rays(sc, cm)
        checked = 0
        for i, r in enumerate(rays):
            k = A._key(r)
            if k not in plus or k not in minus or np.isnan(out["jacobian"][i, 0, k_node]):
                continue
            for col, attr in ((0, "intensity"), (1, "travel_time")):
                fo = getattr(plus[k], attr), getattr(minus[k], attr)
                fd = ((fo[0][0] - fo[1][0]) if col == 0 else (fo[0] - fo[1])) / (2 * h)
                g = out["jacobian"][i, col, k_node]
                assert abs(g - fd) <= 1e-3 * abs(fd) + 1e-9, (k, k_node, col, g, fd)
            checked += 1
        assert checked > 10


def test_torch_function_backward(engine):
    torch = pytest.importorskip("torch")
    sc = A.AdjointScenario(num_de=91, num_az=13, n_steps=160, n_targets=6, max_range=10e3)
    nodes = torch.tensor(A.munk_nodes(), dtype=torch.float64, requires_grad=True)
    bottom = torch.tensor(sc.bottom, dtype=torch.float64, requires_grad=True)
    f = A.EigenrayTLTime
    vals = f.apply(nodes, bottom, sc)
    assert vals.shape[1] == 2 and vals.shape[0] > 3
    w = torch.linspace(0.5, 1.5, vals.shape[0], dtype=torch.float64)
    (vals[:, 0] * w).sum().backward()
    out = A.eigenray_gradients(sc, nodes.detach().numpy())
    jac = np.nan_to_num(out["jacobian"])
    expect = np.einsum("i,ik->k", w.numpy(), jac[:, 0, :])
    assert np.allclose(nodes.grad.numpy(), expect[:20], rtol=1e-9, atol=1e-12)
    assert np.allclose(bottom.grad.numpy(), expect[20:], rtol=1e-9, atol=1e-12)
