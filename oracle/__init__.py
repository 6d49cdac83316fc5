"""TEST INFRASTRUCTURE ONLY: the CPU oracle for the NeMo simulation step.

This package wraps ``libnemo_oracle.so`` (a C restatement of the NeMo 0.7.2
reference CPU backend, built from ``oracle/nemo_oracle.c`` by
``oracle/Makefile``) behind the same Python interface as the product
package ``nemosim_b200`` (which mirrors the reference's Python binding,
src/api/python/nemo_py.cpp:729-816 and src/api/python/__init__.py.in), so a
parity test can drive both with one code path.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package; the product never does.
"""
from .oracle import (  # noqa: F401
    Configuration,
    Network,
    NemoError,
    Simulation,
    build,
    example_random,
    lib,
    nrand,
    seed_states,
    urand,
)
