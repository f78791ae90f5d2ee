"""Helpers for GPU tests: skip cleanly without a device, fail loudly without the library."""
import pytest


def cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def require_gpu():
    if not cuda_available():
        pytest.skip("no CUDA device")
    import aoa_b200.capi as capi
    capi.load()   # raises if libaoa_b200.so is missing: no silent fallback
