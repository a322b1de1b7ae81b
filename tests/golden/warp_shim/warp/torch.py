"""warp.torch stand-in for the golden generator (see warp/__init__.py)."""
import builtins as _b

import warp as _wp


def dtype_from_torch(torch_dtype):
    return _b.int if "int" in str(torch_dtype) else _b.float


def device_from_torch(device):
    return str(device)


def dtype_is_compatible(torch_dtype, warp_dtype):
    return True


def from_torch(t, dtype=None, requires_grad=None, **kw):
    return _wp.from_torch(t, dtype=dtype, requires_grad=requires_grad)
