"""Generates the committed oracle fixtures in this directory.

    python tests/golden/gen_golden.py

Each case runs the CPU oracle (oracle/fx_oracle.c) from a deterministic
initial state and stores the gathered global state.  The fixtures guard the
oracle against regressions; its agreement with the reference algorithm is
established by the known-answer tests in tests/test_oracle.py.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, os.path.join(ROOT, "flash-x_b200"), os.path.dirname(HERE)):
    if p not in sys.path:
        sys.path.insert(0, p)

from flashx_b200 import simulations as S  # noqa: E402
from flashx_b200.params import BC_OUTFLOW, BC_PERIODIC, Geometry, HydroParams  # noqa: E402


def _sod():
    return Geometry(2, 16, 16, 1, 2, 2, 1, bc=(BC_OUTFLOW,) * 6), HydroParams(), S.sod, 1


def _kh():
    return Geometry(2, 16, 16, 1, 2, 2, 1, bc=(BC_PERIODIC,) * 6), HydroParams(), S.kelvin_helmholtz, 3


CASES = {"sod2d_1step": _sod, "kh2d_3step": _kh}


def main():
    from oracle import fx_oracle as O
    from test_oracle import run_oracle
    for name, fn in CASES.items():
        geom, hp, init, nsteps = fn()
        unk = init(geom, hp)
        run_oracle(O, geom, hp, unk, nsteps=nsteps)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), state=S.gather_global(geom, unk))
        print("wrote", name)


if __name__ == "__main__":
    main()
