"""Helpers for GPU tests: numpy uint64 packed matrices <-> torch CUDA tensors."""
import numpy as np
import torch


def to_dev(a: np.ndarray) -> torch.Tensor:
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint64:
        a = a.view(np.int64)
    return torch.from_numpy(a).cuda()


def to_host(t: torch.Tensor) -> np.ndarray:
    a = t.cpu().numpy()
    if a.dtype == np.int64:
        a = a.view(np.uint64)
    return a


def valid_words(a: np.ndarray, n: int) -> np.ndarray:
    """The first ceil(n/64) words of each row (the padding words are not compared)."""
    return a[:, : (n + 63) // 64]
