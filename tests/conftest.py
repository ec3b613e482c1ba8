"""Shared fixtures. Tests marked `gpu` need a CUDA device (B200); everything else runs on
CPU. GPU tests call the runtime only through its C ABI (libparallax-runtime.so)."""
from __future__ import annotations

import ctypes as C
import importlib.util
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs on the B200 box)")


def _load_pkg():
    name = "parallax_runtime_b200"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, ROOT / "parallax-runtime_b200" / "__init__.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def px():
    return _load_pkg()


@pytest.fixture(scope="session")
def lib(px):
    return px.load()


@pytest.fixture(scope="session")
def ox():
    import oracle
    oracle.ox()
    return oracle


class Dev:
    """Device buffers (torch allocations) addressed by raw pointer, like a C caller's."""

    def __init__(self):
        import torch
        assert torch.cuda.is_available(), "gpu tests need a CUDA device"
        self.torch = torch

    def put(self, a: np.ndarray):
        t = self.torch.from_numpy(np.ascontiguousarray(a).view(np.uint8)).cuda()
        return t

    def empty(self, nbytes: int):
        return self.torch.empty(max(nbytes, 1), dtype=self.torch.uint8, device="cuda")

    @staticmethod
    def get(t, dtype, n: int) -> np.ndarray:
        return t[: n * np.dtype(dtype).itemsize].cpu().numpy().view(dtype).copy()


@pytest.fixture(scope="session")
def dev():
    return Dev()


def host_ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def result_buf(nbytes: int = 8):
    return (C.c_ubyte * nbytes)()
