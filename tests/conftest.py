"""Shared pytest setup: markers, import paths and golden-case loading."""
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "metal-route_b200"), os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (run on the B200 box)")


def load_golden():
    with open(os.path.join(ROOT, "tests", "golden", "reference_cases.json")) as f:
        return json.load(f)["cases"]


def case_grid(c):
    from mrcuda.types import Dims, Grid

    dims = Dims(*c["dims"])
    return Grid(
        dims,
        np.array(c["cost"], dtype=np.uint32),
        None if c.get("board") is None else np.array(c["board"], dtype=np.uint8),
        None if c.get("via_forbidden") is None else np.array(c["via_forbidden"], dtype=np.uint8),
    )


def case_nets(c):
    from mrcuda.types import NetEndpoints

    return [NetEndpoints(n["name"], n["src"], n["dst"], list(n["pads"]), list(n["via_pads"])) for n in c["nets"]]


@pytest.fixture(scope="session")
def oracle():
    import oracle as orc

    return orc.get()


@pytest.fixture(scope="session")
def golden():
    return load_golden()
