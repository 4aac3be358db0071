"""Writes tests/golden/ref_<case>.npz: the reference's own example
configurations (tests/ref_fixtures.py) run through the reference-source build
(oracle/_ref, from oracle/build_ref.sh).

Each file holds the particle state as the reference's reader took it from
the example's particle file (in_<field>), the command list (commands, JSON),
and the state after the run (out_<field>), so the parity tests can check the
oracle and the GPU path against the reference's own outputs on a machine
that has neither the reference tree nor its build.

Usage: python tests/golden/make_ref_golden.py [configurations-dir]
       (default /root/reference/configurations)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, os.path.dirname(HERE))

from oracle.refsrc import RefSimulation  # noqa: E402
from ref_fixtures import CASES, INPUT_FIELDS, apply, encode  # noqa: E402


def make(conf_dir: str, name: str) -> str:
    path, box, commands, fields = CASES[name]
    sim = RefSimulation()
    sim.box(*box)
    sim.input_file(os.path.join(conf_dir, path))
    out = {"commands": np.array(encode(commands)), "fields": np.array(" ".join(fields)),
           "box": np.array(box[:3], dtype=np.float64), "periodic": np.array(int(box[3]))}
    for f in INPUT_FIELDS:
        out["in_" + f] = sim.download(f)
    apply(sim, commands)
    for f in fields + ["ix", "iy", "iz"]:
        out["out_" + f] = sim.download(f)
    dest = os.path.join(HERE, f"ref_{name}.npz")
    np.savez_compressed(dest, **out)
    return dest


if __name__ == "__main__":
    conf_dir = sys.argv[1] if len(sys.argv) > 1 else "/root/reference/configurations"
    for name in CASES:
        print(make(conf_dir, name))
