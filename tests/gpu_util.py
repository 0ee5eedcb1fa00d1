"""Helpers for the GPU parity tests: move flat column-major numpy buffers to the device,
call the C-ABI entry points, and bring results back."""
import ctypes

import numpy as np

import rocsolver_b200 as rs


def torch():
    import torch as _t
    return _t


def dev(a):
    t = torch()
    return t.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    torch().cuda.synchronize()
    return t.cpu().numpy()


def ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


class GpuHandle:
    def __init__(self):
        t = torch()
        self.h = rs.Handle(t.cuda.current_stream().cuda_stream)

    @property
    def value(self):
        return self.h.value

    def close(self):
        self.h.close()


def ptr_array(buf, bc, stride):
    """Device array of device pointers to the members of a strided device buffer (for the
    _batched entry points)."""
    t = torch()
    base = buf.data_ptr()
    es = buf.element_size()
    ptrs = np.array([base + b * stride * es for b in range(bc)], dtype=np.uint64)
    return t.from_numpy(ptrs.view(np.int64)).cuda()


def prefix(dtype):
    return "d" if dtype == np.float64 else "s"
