"""The drop-in binary on the reference's own example configurations.

For each example of tests/ref_fixtures.py, `samos_b200/samos-gpu` runs a conf
file with the example's hot-path commands from the state the reference read
(tests/host_examples.py writes both files), and the `dump type=full` it
writes after the run is compared with the state the reference's own code
ended in (tests/golden/ref_*.npz).  Bars: positions within 1e-8 (the 1e-9
trajectory bar plus the dump's 11 significant digits), velocities within
1e-6 relative (8 significant digits printed), directors within 2e-6 (6
decimals printed), image flags exactly.
"""
import glob
import subprocess

import numpy as np
import pytest

from host_examples import BIN, GOLDEN, GOLDEN_IDS, read_full_dump, write_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("path", GOLDEN, ids=GOLDEN_IDS)
def test_host_binary_reproduces_the_reference_example_runs(tmp_path, path):
    if not __import__("os").path.exists(BIN):
        from samos_b200 import build
        build.build_all()
    z = write_case(str(tmp_path), path)
    r = subprocess.run([BIN, "--quiet", "run.conf"], capture_output=True, text=True, timeout=600, cwd=str(tmp_path))
    assert r.returncode == 0, r.stderr[-2000:]
    dumps = sorted(glob.glob(str(tmp_path / "final_*")))
    assert len(dumps) == 1, dumps
    got = read_full_dump(dumps[0])
    for f in str(z["fields"]).split():
        want = z["out_" + f]
        if f in ("x", "y", "z"):
            tol = 1e-8 * max(1.0, float(np.max(np.abs(want))) / 10)
        elif f.startswith("v"):
            tol = 1e-6 * max(1.0, float(np.max(np.abs(want))))
        else:
            tol = 2e-6
        err = float(np.max(np.abs(got[f] - want)))
        assert err <= tol, f"{f}: max |host - reference| = {err}"
    for f in ("ix", "iy"):
        np.testing.assert_array_equal(got[f].astype(int), z["out_" + f], err_msg=f)
