"""Shared test setup: import paths, the `gpu` marker and golden fixtures."""
import json
import pathlib
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
for p in (str(ROOT), str(ROOT / "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU and the built CUDA library")


@pytest.fixture(scope="session")
def certs():
    """{n: (weights float64, meta dict)} for the reference certificates."""
    arr = np.load(GOLDEN / "certificates.npz")
    meta = json.loads((GOLDEN / "certificates.json").read_text())
    return {int(n): (arr[f"w{n}"], meta[n]) for n in meta}


@pytest.fixture(scope="session")
def kat():
    return json.loads((GOLDEN / "kat.json").read_text())


@pytest.fixture(scope="session")
def probe_ls():
    z = np.load(GOLDEN / "probe_ls.npz")
    settings = json.loads(str(z["settings"]))
    return [(s, z[f"start{i}"], z[f"end{i}"]) for i, s in enumerate(settings)]


@pytest.fixture(scope="session")
def orc():
    import oracle
    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def lib():
    import sidon_b200
    return sidon_b200.load(build=True)


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test run without a CUDA device")
    import sidon_b200
    sidon_b200.load(build=True)
    return torch.device("cuda:0")
