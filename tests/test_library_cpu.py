"""CPU-side checks of the C-ABI library: it loads, exports every entry point the
header declares, computes windows like the reference, and fails loudly (never
falls back) when no CUDA device exists."""
import os
import re

import pytest

from conftest import ROOT
import mrcuda
from mrcuda.types import Dims, IsolatedRouteWindow, NetEndpoints


def _declared_symbols():
    with open(os.path.join(ROOT, "include", "mr_cuda.h")) as f:
        text = f.read()
    return sorted(set(re.findall(r"\b(mrc_[a-z_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = mrcuda.load_library()
    declared = _declared_symbols()
    assert len(declared) >= 20
    missing = [name for name in declared if not hasattr(lib, name)]
    assert missing == []


def test_abi_version_matches_header():
    with open(os.path.join(ROOT, "include", "mr_cuda.h")) as f:
        m = re.search(r"#define MRC_ABI_VERSION (\d+)u", f.read())
    assert mrcuda.load_library().mrc_abi_version() == int(m.group(1))


def test_library_windows_match_oracle(oracle):
    import numpy as np

    rng = np.random.default_rng(11)
    for _ in range(50):
        dims = Dims(int(rng.integers(1, 300)), int(rng.integers(1, 300)), int(rng.integers(1, 5)))
        n = len(dims)
        pads = [int(p) for p in rng.integers(0, n, int(rng.integers(0, 4)))]
        net = NetEndpoints("w", int(rng.integers(0, n)), int(rng.integers(0, n)), pads)
        assert mrcuda.net_windows(dims, [net])[0] == oracle.net_window(dims, net)


@pytest.mark.skipif(os.environ.get("CUDA_VISIBLE_DEVICES") is None and os.path.exists("/dev/nvidia0"),
                    reason="a GPU is present; the no-device contract is checked on CPU-only hosts")
def test_no_device_is_an_error_not_a_fallback():
    import torch

    if torch.cuda.is_available():
        pytest.skip("GPU present")
    with pytest.raises(mrcuda.BackendUnavailable):
        mrcuda.Engine(0)
