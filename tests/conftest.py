import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session")
def native():
    """The product library, built in-tree if needed (nvcc cross-compiles without a GPU)."""
    from cvt_b200 import build as pbuild

    pbuild.build()
    from cvt_b200 import _lib

    return _lib.lib()


@pytest.fixture(scope="session")
def orc():
    from oracle import build as obuild
    from oracle.pyoracle import Oracle

    obuild.build_oracle()
    return Oracle("orc")


@pytest.fixture(scope="session")
def ref():
    from oracle import build as obuild
    from oracle.pyoracle import Oracle, available

    obuild.build_ref()
    if not available("ref"):
        pytest.skip("reference kernels not built here (no reference tree, no prebuilt oracle/_ref)")
    return Oracle("ref")


def golden_cases():
    """disparityMap, single level (the reference's setting)"""
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz") and not f.startswith(("pyr", "depth", "vpm", "svpm")))


def pyramid_cases():
    """coarse-to-fine cases (pyramid levels > 1)"""
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz") and f.startswith("pyr"))


def depth_cases():
    """depthMap (the Huber-smoothed variant)"""
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz") and f.startswith("depth"))


def vpm_cases():
    """VPMStereoCL::disparitySimple"""
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz") and f.startswith("vpm"))


def svpm_cases():
    """SVPMFlowCL::flow"""
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz") and f.startswith("svpm"))


def load_golden(name):
    import numpy as np

    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))
