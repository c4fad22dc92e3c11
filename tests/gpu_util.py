"""Helpers for the device tests: torch for device memory, ctypes for the C ABI."""
import ctypes as C

import numpy as np


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def ptr(t):
    return C.c_void_p(t.data_ptr())


def stream():
    import torch
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def sync():
    import torch
    torch.cuda.synchronize()
