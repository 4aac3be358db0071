"""The CUDA path against the reference's own code.

* every scenario of tests/pin_scenarios.py (each potential, aligner,
  external, constraint, integrator and Value kind of the hot path, linear
  temperature schedules and phase-in included), GPU engine against the
  reference-source build (oracle/_ref) run live on the host;
* the reference's example configurations, against the reference's own end
  states stored in tests/golden/ref_*.npz.

Bar: positions, directors and velocities within 1e-9 (the codes differ only
in the last bits of CUDA's sin / cos / exp against glibc's); image flags
identical.  The live comparisons skip when oracle/_ref is not built.
"""
import glob
import os

import numpy as np
import pytest

from oracle import refsrc
from pin_scenarios import NAMES, REFERENCE_UNDEFINED_RUNS, compared_fields, run_backend, run_reference
from samos_b200 import Engine
from test_ref_pin import run_golden_on

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = sorted(glob.glob(os.path.join(HERE, "golden", "ref_*.npz")))
TRAJ = 1e-9


def _close(a, b, what):
    a, b = np.asarray(a, dtype=float), np.asarray(b, dtype=float)
    err = float(np.max(np.abs(a - b))) if a.size else 0.0
    assert err <= TRAJ, f"{what}: max |gpu - reference| = {err}"


@pytest.mark.skipif(not refsrc.available(), reason="reference-source build (oracle/_ref) not built")
@pytest.mark.parametrize("name", [n for n in NAMES if n not in REFERENCE_UNDEFINED_RUNS])
def test_gpu_matches_the_reference_source(name):
    r = run_reference(name)
    e = run_backend(Engine, name)
    for f in compared_fields(name):
        if f in ("ix", "iy", "iz"):
            np.testing.assert_array_equal(e.download(f), r.download(f), err_msg=f"{name}: {f}")
        else:
            _close(e.download(f), r.download(f), f"{name}: {f}")


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[4:-4] for p in GOLDEN])
def test_gpu_reproduces_the_reference_example_runs(path):
    z, e, fields = run_golden_on(Engine, path)
    for f in fields:
        _close(e.download(f), z["out_" + f], f)
    for f in ("ix", "iy"):
        np.testing.assert_array_equal(e.download(f), z["out_" + f], err_msg=f)
