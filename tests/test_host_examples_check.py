"""The conf and particle files that replay the reference's example runs
through `samos-gpu` (tests/host_examples.py), checked without a GPU: every
conf parses and resolves (`--check`), and the particle file reads back as
exactly the state the reference read."""
import os
import subprocess

import numpy as np
import pytest

from host_examples import BIN, COLUMNS, GOLDEN, GOLDEN_IDS, write_case


@pytest.mark.parametrize("path", GOLDEN, ids=GOLDEN_IDS)
def test_example_conf_resolves_and_particles_read_back_exactly(tmp_path, path):
    z = write_case(str(tmp_path), path)
    r = subprocess.run([BIN, "--check", "--quiet", "run.conf"], capture_output=True, text=True, timeout=120,
                       cwd=str(tmp_path))
    assert r.returncode == 0, r.stderr[-2000:]
    n = len(z["in_x"])
    assert f"particles {n} " in r.stdout
    r = subprocess.run([BIN, "--read-particles", os.path.join(str(tmp_path), "p.dat")], capture_output=True,
                       text=True, timeout=120)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = r.stdout.splitlines()
    head = lines[0].split()
    rows = [l.split() for l in lines[1:]]
    assert len(rows) == n
    for c in COLUMNS:
        k = head.index(c)
        got = np.array([float(row[k]) for row in rows])
        np.testing.assert_array_equal(got, np.asarray(z["in_" + c], dtype=float), err_msg=c)
