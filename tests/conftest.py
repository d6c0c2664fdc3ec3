"""Shared fixtures.  `-m gpu` tests need a B200 and the in-tree libmpgpu.so;
everything else runs on CPU."""
from __future__ import annotations

import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 GPU and the built CUDA library")


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle, build
    if not os.path.exists(os.path.join(ROOT, "oracle", "libscrimp_oracle.so")):
        build(with_reference=False)
    return Oracle()


@pytest.fixture(scope="session")
def golden_ascii():
    return dict(np.load(os.path.join(GOLDEN, "test_ascii.npz")))


@pytest.fixture(scope="session")
def golden_edges():
    z = np.load(os.path.join(GOLDEN, "edge_cases.npz"))
    cases = {}
    for k in z.files:
        name, field = k.split("__")
        cases.setdefault(name, {})[field] = z[k]
    return cases


@pytest.fixture(scope="session")
def golden_prescrimp():
    """The reference's PreSCRIMP outputs (tests/golden/make_prescrimp_golden.py):
    {case: {"x", "m", "stride", "dist" (sqrt |d2|), "index", "exact_dist", "exact_index"}};
    dist/index are PreSCRIMP's profile, exact_* the final SCRIMP++ profile."""
    z = np.load(os.path.join(GOLDEN, "prescrimp_ref.npz"))
    cases = {}
    for name in z["names"]:
        cases[str(name)] = {f: z[f"{name}/{f}"] for f in ("x", "m", "stride", "dist", "index",
                                                           "exact_dist", "exact_index")}
    return cases


@pytest.fixture(scope="session")
def digests():
    return json.load(open(os.path.join(GOLDEN, "digests.json")))


@pytest.fixture(scope="session")
def gpu_ctx():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("gpu test on a host without CUDA")
    import thesiscode_b200 as mp
    ctx = mp.Context(0)
    yield ctx
    ctx.close()
