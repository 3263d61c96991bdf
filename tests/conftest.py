import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    # Build the product library and the oracle in-tree when they are missing (they are built
    # artefacts: a prebuilt working tree already holds them).
    lib = os.path.join(ROOT, "supertrack_b200", "libsupertrack_b200.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-C", os.path.join(ROOT, "supertrack_b200"), "-j8"], check=True)
    olib = os.path.join(ROOT, "oracle", "liboracle.so")
    if not os.path.exists(olib):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True)


@pytest.fixture(scope="session")
def ctx():
    """One GPU context for the GPU tests of a session."""
    import supertrack_b200 as st
    c = st.Context(0)
    yield c
    c.close()
