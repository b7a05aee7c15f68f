"""Shared fixtures: seeded AWSIM set-ups written to a temporary directory, the parsed
configuration and its fields, and helpers that build the CPU oracle on demand."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    oracle.build(ref=True)
    return oracle


def make_setup(tmp, kind, **kw):
    from pawsim_b200 import inputs
    fn = {"gyre": inputs.gyre, "channel": inputs.channel, "jets": inputs.jets,
          "full": inputs.full_physics}[kind]
    path = fn(os.path.join(str(tmp), kind), **kw)
    cfg = inputs.read_config(path)
    return path, cfg, inputs.load_fields(cfg)


def value_equal(a, b):
    """Bit-exact comparison up to the sign of zero (IEEE equality, NaN never equal)."""
    return bool(np.array_equal(np.asarray(a), np.asarray(b)))


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    d = np.linalg.norm(a - b)
    n = np.linalg.norm(b)
    return d / n if n > 0 else d
