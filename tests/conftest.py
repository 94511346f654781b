"""Test configuration: the `gpu` marker and in-tree native builds.

`-m "not gpu"` tests need no GPU: they check the oracle against the golden
vectors, the geometry generator, the host-side table builder and that the
C-ABI library loads and exports every declared symbol.  `-m gpu` tests run
the CUDA solver through the C-ABI and compare it with the oracle and the
golden vectors.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    # Build the native libraries in-tree when they are missing (no-op otherwise).
    from licom4py_gpu_b200 import build
    for lib, fn in (("libduogrid.so", build.build_duogrid), ("libbt.so", build.build_bt)):
        if not os.path.exists(os.path.join(build.LIBDIR, lib)):
            fn()


def load_golden(name):
    import numpy as np
    with np.load(os.path.join(GOLDEN, name)) as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="session")
def grids():
    """Generated geometry per resolution (cached for the session)."""
    from licom4py_gpu_b200 import duogrid_gen
    cache = {}

    def get(n):
        if n not in cache:
            cache[n] = duogrid_gen.generate(n)
        return cache[n]
    return get
