import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    # Build the test oracles (the compiled reference needs the reference tree,
    # the C restatement does not); prebuilt libraries are used as they are.
    subprocess.run(["make", "-s", "-C", str(ROOT / "oracle")], check=False, capture_output=True)


def _have_ref() -> bool:
    return (ROOT / "oracle" / "_ref" / "libgelios_ref.so").exists()


@pytest.fixture(scope="session")
def have_ref():
    if not _have_ref():
        pytest.skip("compiled reference (oracle/_ref/libgelios_ref.so) not available")
    return True


@pytest.fixture(autouse=True)
def _single_thread_reference(monkeypatch):
    # parity runs of the reference use one OpenMP thread: its multithreaded
    # dt reduction is racy (Setka.cpp:10141, 10359-10393)
    monkeypatch.setenv("OMP_NUM_THREADS", "1")
