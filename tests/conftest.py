import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the product's kernels")


def pytest_collection_modifyitems(config, items):
    # The no-allocation entry-point test file runs last so that a stop-at-first-
    # failure run has already run everything else.
    items.sort(key=lambda it: 1 if os.path.basename(str(it.fspath)).startswith("test_zz_") else 0)


@pytest.fixture(scope="session")
def port():
    from oracle.oracle import Port
    return Port()


@pytest.fixture(scope="session")
def reference():
    from oracle.oracle import Reference, reference_available
    if not reference_available():
        pytest.skip("SORT reference library (oracle/_ref) not built on this machine")
    return Reference()


def golden(name):
    import numpy as np
    return np.load(os.path.join(ROOT, "tests", "golden", f"{name}.npz"))


def same_bits(a, b):
    import numpy as np
    a = np.asarray(a)
    b = np.asarray(b)
    return a.shape == b.shape and np.array_equal(a.view(np.int32), b.view(np.int32))


def renumber_topology(topo, new_id):
    """The pre-order topology stream (interior [cnt, children...], leaf
    [0, cnt, ids...]) with every primitive id p replaced by new_id[p]."""
    import numpy as np
    topo = np.asarray(topo)
    out = topo.copy()
    new_id = np.asarray(new_id)
    k = 0

    def walk():
        nonlocal k
        cnt = int(topo[k])
        k += 1
        if cnt == 0:
            n = int(topo[k])
            k += 1
            out[k:k + n] = new_id[topo[k:k + n]]
            k += n
            return
        for _ in range(cnt):
            walk()

    if topo.size:
        walk()
    return out
