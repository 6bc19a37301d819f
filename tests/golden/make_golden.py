"""Generate tests/golden/oracle_small.npz: the oracle's state after a few RK3 steps on the reference's three
18 x 17 x 18 regression grids (tests/regression/{tgv_small,chan_small,chan_les_amd_small}/input_parameters) with
this repository's seeded initial conditions.  The reference itself cannot be built here, so these fixtures pin
the restatement against accidental change; they are not reference outputs.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "dopamine-fdm_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as O  # noqa: E402
from dfdm import cases  # noqa: E402

STEPS = 5


def main():
    O.build()
    out = {}
    for name in ("tgv_small", "chan_small", "chan_les_amd_small"):
        c = cases.get(name)
        o = O.Oracle(c)
        U, V, W, P = cases.initial_condition(c)
        o.set_state(U, V, W, P)
        o.step(STEPS)
        U, V, W, P = o.get_state()
        out[f"{name}_steps"] = np.array(STEPS)
        for k, a in (("U", U), ("V", V), ("W", W), ("P", P)):
            out[f"{name}_{k}"] = a
    np.savez_compressed(os.path.join(HERE, "oracle_small.npz"), **out)


if __name__ == "__main__":
    main()
