"""The bounds-checked build (libwq3d_checked.so, WQ3D_CHECKED=1): every
index a kernel reads from device data is tested before use.  On the
workloads below no test may fire (a failed one ends the run with an
internal error) and the results must equal the default build's bit for
bit.  The checked build runs in a child process, since a process loads one
engine library."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import hashlib, json, sys
import underseamodelinglibrary_b200 as u
from underseamodelinglibrary_b200 import _abi, scenarios as S

def digest(sc, precision, schedule):
    q = S.build_queue(sc, u.wave_queue, precision=precision)
    q.set_reflect_schedule(schedule)
    q.run(sc["time_max"])
    rays = q.take_eigenrays()
    h = hashlib.sha1()
    for r in rays:
        h.update(repr((r.step, r.t1, r.t2, r.de_index, r.az_index, r.travel_time,
                       [float(x) for x in r.intensity], [float(x) for x in r.phase],
                       r.surface, r.bottom, r.caustic)).encode())
    f = q.curr()
    h.update(f.rho.tobytes() + f.theta.tobytes() + f.phase.tobytes() + f.caustic.tobytes())
    return [len(rays), h.hexdigest()]

cases = [
    (S.linear_slope_rayleigh(num_de=181, num_az=19, n_range=8, n_depth=8, time_max=12.0), _abi.FP32C),
    (S.linear_slope_rayleigh(num_de=181, num_az=19, n_range=8, n_depth=8, time_max=12.0), _abi.FP64),
    (S.gridded_munk(seed=5, num_de=121, num_az=13, time_max=12.0, dt=0.05), _abi.FP32C),
    (S.eigenray_basic(), _abi.FP64),
]
out = {"lib": _abi.LIB_PATH, "runs": []}
for sc, prec in cases:
    for sched in (_abi.REFLECT_SIDE, _abi.REFLECT_INLINE):
        out["runs"].append(digest(sc, prec, sched))
print(json.dumps(out))
"""


def _run(env_lib):
    env = dict(os.environ)
    env.pop("WQ3D_LIBRARY", None)
    if env_lib:
        env["WQ3D_LIBRARY"] = env_lib
    env["PYTHONPATH"] = ROOT + os.pathsep + env.get("PYTHONPATH", "")
    p = subprocess.run([sys.executable, "-c", SCRIPT], env=env, cwd=ROOT, capture_output=True, text=True,
                       timeout=600)
    assert p.returncode == 0, p.stderr[-3000:]
    return json.loads(p.stdout.strip().splitlines()[-1])


def test_checked_build_matches_default_build(engine):
    checked = _run("checked")
    plain = _run(None)
    assert checked["lib"].endswith("libwq3d_checked.so")
    assert plain["lib"].endswith("libwq3d.so")
    assert checked["runs"] == plain["runs"]
    assert sum(n for n, _ in plain["runs"]) > 0
