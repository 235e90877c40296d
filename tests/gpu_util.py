"""Helpers for GPU tests: torch views of library-owned device memory."""


class _Raw:
    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (int(ptr), False),
                                         "version": 3}


def device_view(ptr, n):
    """torch float64 view of n doubles at a raw device address owned by the library."""
    import torch
    return torch.as_tensor(_Raw(ptr, n), device="cuda")
