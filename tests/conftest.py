import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libcsdecomp_b200.so")


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(GOLDEN, "golden.json")) as f:
        return json.load(f)


class GoldenPlant:
    def __init__(self, npz, name):
        from csdecomp_b200.plant import MinimalPlant
        keys = [k.split("/", 1)[1] for k in npz.files if k.startswith(name + "/")]
        a = {k: npz[f"{name}/{k}"] for k in keys}
        J, L, D, G, P = [int(x) for x in a["meta"]]
        self.plant = MinimalPlant.from_arrays(a, D, L)
        self.lower = a["lower"]
        self.upper = a["upper"]
        self.robot_geometry_ids = [int(x) for x in a["robot_geometry_ids"]]
        self.link_names = [str(x) for x in a["link_names"]]
        self.dim = D

    def link(self, name):
        return self.link_names.index(name)


@pytest.fixture(scope="session")
def plants():
    npz = np.load(os.path.join(GOLDEN, "plants.npz"))
    names = sorted({k.split("/")[0] for k in npz.files})
    return {n: GoldenPlant(npz, n) for n in names}
