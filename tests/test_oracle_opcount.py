"""Operation counts of the reference algorithm, from the oracle built with
a counting scalar type (oracle/opcount.cpp): the FP64 work of one ray step
(AB3, wave_front::update, reflection and caustic tests; the reference's
wave_queue::step, wave_queue.cc:156-190), of one target distance
(wave_front::compute_target_distance, wave_front.cc:222-236), of the CPA
search per ray and target (wave_queue.cc:351-488), and of one eigenray
construction (wave_queue.cc:495-977 with spreading_hybrid_gaussian).

Run as a script, it prints the counts for the plain FP64 Munk workload
(181 x 37 rays, 100 targets, 60 s) and for the sloped Rayleigh workload's
full D/E fan on 6 AZ columns:
    python tests/test_oracle_opcount.py
"""
import ctypes as C
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

from oracle_binding import OracleQueue, load_oracle  # noqa: E402
from underseamodelinglibrary_b200 import scenarios as S  # noqa: E402
from underseamodelinglibrary_b200 import types as T  # noqa: E402

PHASES = ("step", "target_distance", "cpa_search", "eigenray_build")
KINDS = ("add", "mul", "div", "sqrt", "math", "cmp")


def read_counts(lib):
    buf = (C.c_uint64 * 24)()
    lib.oracle_opcount_read(buf)
    return np.array(buf, dtype=np.float64).reshape(4, 6)


def count_run(sc, steps):
    """operation counts of ``steps`` steps (the constructor's start-up
    excluded), the ray count and the eigenrays found"""
    lib = load_oracle(opcount=True)
    q = S.build_queue(sc, OracleQueue, opcount=True)
    lib.oracle_opcount_reset()
    q.step(steps)
    c = read_counts(lib)
    nrays = sc["de"].size() * sc["az"].size()
    return c, nrays, len(q.take_eigenrays())


def per_unit(sc, steps):
    """FP64 operations per unit: per ray-step, per ray-step-target, per
    eigenray; 'flops' counts add, mul, div and sqrt as one each"""
    c, nrays, neig = count_run(sc, steps)
    nt = sc["targets"].size1() * sc["targets"].size2() if sc["targets"] is not None else 0
    rs = float(nrays) * steps
    out = {"rays": nrays, "steps": steps, "targets": nt, "eigenrays": neig}
    for p, name in enumerate(PHASES):
        unit = {"step": rs, "target_distance": rs * nt, "cpa_search": rs * nt,
                "eigenray_build": max(neig, 1)}[name]
        out[name] = {k: c[p, j] / unit for j, k in enumerate(KINDS)}
        out[name]["flops"] = sum(c[p, j] for j in range(4)) / unit
    return out


def test_counting_build_matches_the_oracle():
    """the counting build computes what the oracle computes"""
    sc = S.munk_flat(num_de=31, num_az=9, n_targets=3, time_max=20.0)
    a = S.build_queue(sc, OracleQueue)
    b = S.build_queue(sc, OracleQueue, opcount=True)
    a.step(150)
    b.step(150)
    ra, rb = a.take_eigenrays(), b.take_eigenrays()
    assert len(ra) > 0 and len(ra) == len(rb)
    for x, y in zip(ra, rb):
        assert x.travel_time == y.travel_time and np.array_equal(x.intensity, y.intensity)


def test_step_and_target_counts():
    """the counts per ray step and per target are properties of the
    algorithm: independent of the fan size, and the target distance is the
    closed form's fixed sequence of operations"""
    a = per_unit(S.munk_flat(num_de=31, num_az=9, n_targets=3, time_max=20.0), 100)
    b = per_unit(S.munk_flat(num_de=61, num_az=13, n_targets=3, time_max=20.0), 100)
    for k in ("flops", "math"):
        assert abs(a["step"][k] - b["step"][k]) <= 0.02 * a["step"][k], (k, a["step"], b["step"])
    assert a["target_distance"]["flops"] == b["target_distance"]["flops"]
    assert 10 <= a["target_distance"]["flops"] <= 40
    assert 50 <= a["step"]["flops"] <= 1000


def _report():
    rows = [("plain FP64 Munk workload, 181 x 37 rays, 100 targets, 600 steps",
             S.munk_flat(), 600),
            ("sloped Rayleigh workload, 1801 D/E x 6 AZ columns, 1024 targets, 200 steps",
             None, 200)]
    for title, sc, steps in rows:
        if sc is None:
            sc = S.linear_slope_rayleigh(num_de=1801, num_az=91, time_max=40.0)
            sc["az"] = T.seq_linear(0.0, 4.0, 6)
        r = per_unit(sc, steps)
        print(title)
        print("  rays %d, steps %d, targets %d, eigenrays %d" % (r["rays"], r["steps"], r["targets"],
                                                              r["eigenrays"]))
        for name, unit in (("step", "ray-step"), ("target_distance", "ray-step-target"),
                           ("cpa_search", "ray-step-target"), ("eigenray_build", "eigenray")):
            d = r[name]
            print("  %-16s per %-16s flops %10.2f  (add %.2f mul %.2f div %.2f sqrt %.2f) math %.2f cmp %.2f"
                  % (name, unit, d["flops"], d["add"], d["mul"], d["div"], d["sqrt"], d["math"], d["cmp"]))


if __name__ == "__main__":
    _report()
