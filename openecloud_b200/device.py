"""Device plumbing: torch supplies device memory and the current CUDA stream.

The compute itself is in liboec.so; nothing here falls back to the CPU.
"""
import numpy as np
import torch

_DEV = None


def device():
    """The CUDA device used by the package (raises when no GPU is visible)."""
    global _DEV
    if _DEV is None:
        if not torch.cuda.is_available():
            raise RuntimeError("openecloud_b200 needs a CUDA device (sm_100a); none is visible")
        _DEV = torch.device("cuda", torch.cuda.current_device())
    return _DEV


def stream():
    """Handle of the current torch CUDA stream, as the C ABI's void* stream."""
    return torch.cuda.current_stream(device()).cuda_stream


def ptr(t):
    return t.data_ptr() if t is not None else None


def empty(shape, dtype):
    return torch.empty(shape, dtype=dtype, device=device())


def zeros(shape, dtype):
    return torch.zeros(shape, dtype=dtype, device=device())


def to_device(a, dtype=torch.float64):
    """numpy / list / tensor -> contiguous device tensor of `dtype`."""
    if isinstance(a, torch.Tensor):
        return a.to(device=device(), dtype=dtype).contiguous()
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype).to(device()).contiguous()


def to_numpy(t):
    if isinstance(t, torch.Tensor):
        return t.detach().cpu().numpy()
    return np.asarray(t)


def round_up(n, m):
    return ((int(n) + m - 1) // m) * m
