import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running")


def _ensure_oracle_built():
    so = os.path.join(ROOT, "oracle", "_build", "libdt_oracle.so")
    if not os.path.exists(so):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "_build/libdt_oracle.so"],
                       check=True)


@pytest.fixture(scope="session")
def oracle_sparse():
    _ensure_oracle_built()
    from oracle import sparse
    return sparse


@pytest.fixture(scope="session")
def oracle_ref():
    from oracle import ref
    if not ref.available():
        # oracle/Makefile builds it where the reference sources are present
        # (REF, overridable by $DIANA_REF) and is a no-op elsewhere.
        cmd = ["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref"]
        if os.environ.get("DIANA_REF"):
            cmd.append("REF=" + os.environ["DIANA_REF"])
        subprocess.run(cmd, check=True)
    if not ref.available():
        pytest.skip("compiled reference oracle (oracle/_ref/libdiana_ref.so) not available")
    return ref


@pytest.fixture(scope="session")
def ctx():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from diana_tucker_b200 import Context
    c = Context(0)
    yield c
    c.close()
