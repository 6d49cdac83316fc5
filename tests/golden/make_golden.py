"""Writes the golden vectors of tests/golden/ from the oracle.

    python tests/golden/make_golden.py

rng.npz         seeds of local indices 0..63 and 1000..1063
                (src/nemo/RNG.cpp:38-63) and 64 nrand draws per seed
                (src/nemo/RNG.cpp:25-33, host glibc logf/sinf)
random_1k.npz   random::construct(1000, 100, 20, false), 1000 ms: per-step
                fired counts, fired ids, final (u, v)
stdp_2k.npz     random::construct(2000, 200, 20, true) with the standard
                STDP window, 500 ms, applyStdp(1.0) every 100 ms: per-step
                counts, fired ids, all weights (Q11.20)

The vectors freeze the oracle's output so that a later change of the oracle
(or of the host libm it calls) shows up as a failing test.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle as O  # noqa: E402
from tests import nets  # noqa: E402


def main():
    seeds0 = O.seed_states(0, 64)
    seeds1000 = O.seed_states(1000, 64)
    out = np.zeros((64, 64), np.float32)
    for i in range(64):
        s = seeds0[i].copy()
        for k in range(64):
            out[i, k] = O.nrand(s)
    np.savez_compressed(os.path.join(HERE, "rng.npz"), seeds0=seeds0, seeds1000=seeds1000, nrand=out)

    sim = O.Simulation(O.example_random(1000, 100, 20, False), O.Configuration())
    counts, ids = sim.run(1000)
    np.savez_compressed(os.path.join(HERE, "random_1k.npz"), counts=counts, ids=ids,
                        state=sim.type_state(0, 2, 1000))

    sim = O.Simulation(O.example_random(2000, 200, 20, True), nets.standard_stdp(O))
    counts, ids = sim.run(500, 100, 1.0)
    np.savez_compressed(os.path.join(HERE, "stdp_2k.npz"), counts=counts, ids=ids,
                        weights=sim.weights_fx(2000 * 200))
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main()
