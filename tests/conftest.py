import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

# The reference source tree the checkers under oracle/_ref are built from
# (the same variable oracle/Makefile reads); absent on machines that only
# run the prebuilt checkers.
REFERENCE_SRC = os.path.join(os.environ.get("REFERENCE", "/root/reference"), "src")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: longer CPU or GPU runs")


def _ensure_checkers():
    """Builds the oracle (and, where the reference sources exist, the
    reference checkers) if they are missing."""
    oracle_so = os.path.join(ROOT, "oracle", "libmpd_oracle.so")
    if not os.path.exists(oracle_so):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    ref_so = os.path.join(ROOT, "oracle", "_ref", "libref_byte8.so")
    if not os.path.exists(ref_so) and os.path.isdir(REFERENCE_SRC):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True)


_ensure_checkers()


def cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu():
    if not cuda_available():
        pytest.skip("no CUDA device")
    return 0
