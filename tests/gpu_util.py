"""Helpers shared by the GPU tests (skip cleanly without a device)."""
import numpy as np
import pytest


def need_gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def relerr(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(1e-300, np.max(np.abs(b))))


def device_array(torch, ptr, n, typestr="<f8"):
    """Host copy of n elements at a device pointer of this library (read
    through the CUDA array interface)."""
    class _View:
        __cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (int(ptr), False), "version": 3}
    torch.cuda.synchronize()
    return torch.as_tensor(_View(), device="cuda").cpu().numpy()
