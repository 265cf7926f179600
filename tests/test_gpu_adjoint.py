"""Gradients of eigenray TL and travel time (underseamodelinglibrary_b200
.adjoint) against central differences of the CPU oracle (the FP64
restatement of the reference): the engine's reverse sweep for the
sound-speed nodes, the exact bottom-parameter derivatives of the
sensitivity mode, and the torch.autograd.Function wrapper.

Difference steps.  A step of 1e-3 of a node's sound speed (1.5 m/s) is
outside the linear range of many rays: near the sound-channel axis the
difference quotient at that step is tens of percent away from its limit,
and about a third of the eigenrays change their (step, target, D/E, AZ)
bracket under it.  Small steps meet rounding instead: an eigenray's
travel time comes from a Taylor fit to distance^2 values of about 1e8 m^2
formed as differences of 4e13 m^2 terms, so the quotient's noise grows
like 1e-8 / h (1 % at h = 1e-6 c_k).  The oracle's differences are
therefore taken at 1e-4 and 5e-5 of c_k and extrapolated (Richardson:
(4 D(h/2) - D(h)) / 3).  An (eigenray, node) pair is checked where its
bracket holds at both steps and the two quotients agree within 2e-3 (the
steps resolve the derivative).  There the adjoint must agree with the
extrapolation within 1e-3 plus the two quotients' own spread (the
difference's uncertainty) on at least 95 % of the pairs, and within 2e-2
on all of them (the worst pairs seen, about 1.5e-2, are travel-time rows
of steep eigenrays beside a bottom bounce, where the offset fit takes its
clamped branches); an absolute floor of 1e-6 dB or 1e-9 s per m/s
applies."""
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from underseamodelinglibrary_b200 import adjoint as A
from oracle_binding import OracleQueue, load_oracle

pytestmark = pytest.mark.gpu

REL = 1e-3
AGREE = 2e-3
H1, H2 = 1e-4, 5e-5
FLOORS = (1e-6, 1e-9)


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
    """the oracle's eigenrays with node k moved by +-h c_k, for both steps
    (the runs go to a thread pool: the oracle's calls release the GIL)"""
    sc, nodes, _ = prop
    load_oracle()
    jobs = [(k, hr, sgn) for k in range(nodes.size) for hr in (H1, H2) for sgn in (1, -1)]

    def run(job):
        k, hr, sgn = job
        c = nodes.copy()
        c[k] += sgn * hr * abs(nodes[k])
        return job, oracle_rays(sc, c)

    with ThreadPoolExecutor(max_workers=max(1, min(32, os.cpu_count() or 1))) as ex:
        return dict(ex.map(run, jobs))


def differences(res, nodes, key, k, hr):
    """(d TL, d T) / d c_k of one eigenray at step hr, or None when its
    bracket does not hold under both moves"""
    h = hr * abs(nodes[k])
    p, m = res[(k, hr, 1)], res[(k, hr, -1)]
    if key not in p or key not in m:
        return None
    return ((p[key].intensity[0] - m[key].intensity[0]) / (2 * h),
            (p[key].travel_time - m[key].travel_time) / (2 * h))


def resolved(a, b, j):
    return a is not None and b is not None and \
        abs(a[j] - b[j]) <= AGREE * max(abs(a[j]), abs(b[j])) + FLOORS[j]


def extrapolated(a, b):
    """Richardson's extrapolation of central differences at h and h/2"""
    return (4.0 * b - a) / 3.0


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


@pytest.fixture(scope="module")
def sampled_rows(prop):
    """Jacobian rows of 16 random eigenrays (two unit-weight sweeps each)"""
    sc, nodes, p = prop
    rng = np.random.default_rng(7)
    idx = sorted(rng.choice(len(p.eigenrays), size=min(16, len(p.eigenrays)), replace=False))
    return idx, p.rows(idx)


def test_adjoint_rows_match_oracle_differences(prop, oracle_fd, sampled_rows):
    """Jacobian rows from unit-weight reverse sweeps against the oracle's
    extrapolated central differences, node by node, wherever the steps
    resolve the derivative"""
    sc, nodes, p = prop
    rays = p.eigenrays
    idx, rows = sampled_rows
    errs, total = [], 0
    for r_i, i in enumerate(idx):
        key = A._key(rays[i])
        for k in range(nodes.size):
            a = differences(oracle_fd, nodes, key, k, H1)
            b = differences(oracle_fd, nodes, key, k, H2)
            for j in (0, 1):
                total += 1
                if not resolved(a, b, j):
                    continue
                want = extrapolated(a[j], b[j])
                g = rows[r_i, j, k]
                scale = max(abs(want), FLOORS[j] / REL)
                # error beyond the differences' own spread, relative
                errs.append((max(0.0, abs(g - want) - abs(a[j] - b[j])) / scale, key, k, j, g, want))
    assert len(errs) >= 0.6 * total, (len(errs), total)
    rel = np.array([e[0] for e in errs])
    worst = max(errs)
    assert np.mean(rel <= REL) >= 0.95, (np.mean(rel <= REL), np.percentile(rel, [50, 90, 99]), worst)
    assert worst[0] <= 20 * REL, worst


def test_vjp_is_the_weighted_sum_of_rows(prop, sampled_rows):
    """one reverse sweep with weights on several eigenrays equals the same
    weighted sum of their unit-weight rows (the sweep is linear in its
    seeds), and the bottom part is the weighted exact sensitivities"""
    sc, nodes, p = prop
    idx, rows = sampled_rows
    n = len(p.eigenrays)
    rng = np.random.default_rng(11)
    w_tl, w_t = np.zeros(n), np.zeros(n)
    w_tl[idx] = rng.normal(size=len(idx))
    w_t[idx] = rng.normal(size=len(idx)) * 1000.0
    g, gb, ms = p.vjp(w_tl, w_t)
    assert ms > 0.0
    want = w_tl[idx] @ rows[:, 0, :nodes.size] + w_t[idx] @ rows[:, 1, :nodes.size]
    assert np.allclose(g, want, rtol=1e-9, atol=1e-12 * np.abs(want).max())
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
