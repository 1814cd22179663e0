"""Regenerates the golden fixtures from the reference's own CPU engine.

    python tests/golden/make_golden.py

Needs oracle/_ref/libspref.so, i.e. the reference sources at build time
(`make -C oracle ref`).  Each fixture holds the scenario's inputs and the
reference's outputs (iterates, pixel flags, iteration count, Fourier and
real-space errors, support fraction); scenarios are in scenarios.py.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

import oracle  # noqa: E402
import scenarios  # noqa: E402


def main():
    oracle.build(ref=True)
    for name in scenarios.SCENARIOS:
        amp, mask, support = scenarios.inputs(name)
        eng = oracle.Reference(scenarios.SCENARIOS[name]["shape"])
        out = scenarios.run(eng, name, amp, mask, support)
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, amp=amp, mask=mask, support=support, **out)
        print(f"{path}: iteration {int(out['iteration'])} efourier {float(out['efourier']):.6g}")


if __name__ == "__main__":
    main()
