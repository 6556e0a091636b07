"""PDF and flag fields as PyTorch CUDA tensors in lbmpy's layout.

lbmpy stores a PDF field as an array of shape ``(X+2, Y+2, Z+2, Q)`` (one ghost layer) with the
'fzyx' memory layout: x fastest, the PDF index slowest (``updatekernels.py:146-163``,
``creationfunctions.py:605-618``).  ``create_pdf_array`` returns exactly that view, with rows
padded so that the first interior cell of every row starts on a 32-byte sector boundary; the
padding is invisible through the view.
"""
from __future__ import annotations

import torch

# e3m12 (1 sign, 3 exponent, 12 mantissa bits, scaled by 16; include/lbm_b200.h) has no torch type:
# its 16-bit codes live in an int16 tensor
_TORCH_DTYPES = {"float64": torch.float64, "float32": torch.float32, "float16": torch.float16,
                 "bfloat16": torch.bfloat16, "e3m12": torch.int16}
ALIGN_BYTES = 32


def torch_dtype(name: str):
    return _TORCH_DTYPES[name]


def dtype_name(dt: torch.dtype) -> str:
    for k, v in _TORCH_DTYPES.items():
        if v == dt:
            return k
    raise ValueError(f"unsupported PDF dtype {dt}")


def create_pdf_array(size, num_directions, ghost_layers=1, layout="fzyx", dtype="float64", device="cuda",
                     fill=0.0):
    """Zero-filled PDF tensor of shape ``size + 2*ghost_layers`` plus ``(num_directions,)``."""
    if ghost_layers != 1:
        raise NotImplementedError("the B200 sweep uses exactly one ghost layer")
    if layout not in ("fzyx", "f", "reverse_numpy", "SoA"):
        raise NotImplementedError("only the fzyx (SoA) layout is supported")
    size = tuple(int(s) for s in size)
    if len(size) != 3:
        raise ValueError("the B200 sweep is three-dimensional: size must have three entries")
    tdt = dtype if isinstance(dtype, torch.dtype) else _TORCH_DTYPES[str(dtype)]
    itemsize = torch.tensor([], dtype=tdt).element_size()
    a = max(1, ALIGN_BYTES // itemsize)
    ex, ey, ez = size[0] + 2, size[1] + 2, size[2] + 2
    sy = -(-ex // a) * a
    sz = sy * ey
    sq = sz * ez
    off = a - 1                        # element x=1 of every row lands on an aligned address
    buf = torch.full((off + num_directions * sq,), fill, dtype=tdt, device=device)
    return torch.as_strided(buf, (ex, ey, ez, num_directions), (1, sy, sz, sq), off)


def pdf_strides(t: torch.Tensor):
    if t.dim() != 4:
        raise ValueError(f"PDF field must have 4 dimensions (x, y, z, q), got shape {tuple(t.shape)}")
    return tuple(int(s) for s in t.stride())


def check_pdf_tensor(t: torch.Tensor, q: int, dtype_name_: str, name: str = "pdfs"):
    if not isinstance(t, torch.Tensor):
        raise TypeError(f"{name} must be a torch tensor")
    if not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor (the B200 sweep has no CPU path)")
    if t.dim() != 4 or t.shape[3] != q:
        raise ValueError(f"{name} must have shape (X+2, Y+2, Z+2, {q}), got {tuple(t.shape)}")
    if dtype_name(t.dtype) != dtype_name_:
        raise ValueError(f"{name} has dtype {t.dtype}, the kernel was built for {dtype_name_}")
    if t.stride(0) != 1:
        raise ValueError(f"{name} must have the fzyx layout (x stride 1), got strides {t.stride()}")


def create_flag_array(size, device="cuda"):
    """uint8 cell flags over the ghost-inclusive domain, x fastest (see include/lbm_b200.h)."""
    ex, ey, ez = (int(s) + 2 for s in size)
    return torch.zeros((ez, ey, ex), dtype=torch.uint8, device=device).permute(2, 1, 0)
