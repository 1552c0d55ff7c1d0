import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
# the float64 reference of the differentiable form (oracle/lif_reference.py)
if os.path.join(ROOT, "oracle") not in sys.path:
    sys.path.insert(0, os.path.join(ROOT, "oracle"))

ORACLE_LIB = os.path.join(ROOT, "oracle", "_build", "libnemo_oracle.so")
ORACLE_REF_DIR = os.path.join(ROOT, "oracle", "_ref")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 (runs the sm_100a library)")
    config.addinivalue_line("markers", "slow: long-running CPU case")


def ensure_oracle():
    """Build the oracle (test infrastructure) if it is missing."""
    if not os.path.exists(ORACLE_LIB):
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle")])
    return ORACLE_LIB


@pytest.fixture(scope="session")
def oracle_lib():
    from nemo_b200.nemo import Library
    return Library(ensure_oracle())


@pytest.fixture(scope="session")
def b200_lib():
    from nemo_b200.nemo import Library
    return Library()  # the product library; fails loudly if it is not built


@pytest.fixture(params=["oracle", pytest.param("b200", marks=pytest.mark.gpu)])
def lib(request):
    """Run a known-answer test against the oracle (CPU) and the B200 library."""
    from nemo_b200.nemo import Library
    if request.param == "oracle":
        return Library(ensure_oracle())
    return Library()


def configuration(lib, stdp=False, backend="default"):
    """src/test/utils.cpp:83-103: the standard test configuration; with STDP
    the function pre[i]=0.1*exp(-(i+1)/20), post[i]=-0.08*exp(-(i+1)/20) and
    limits (-10, 10)."""
    import numpy as np
    from nemo_b200.nemo import Configuration
    conf = Configuration(lib)
    if stdp:
        dt = np.arange(1, 21, dtype=np.float32)
        pre = (np.float32(0.1) * np.exp(-dt / np.float32(20.0))).astype(np.float32)
        post = (np.float32(-0.08) * np.exp(-dt / np.float32(20.0))).astype(np.float32)
        conf.set_stdp_function(pre, post, -10.0, 10.0)
    if lib.path == ORACLE_LIB:
        conf.set_cpu_backend()
    return conf
