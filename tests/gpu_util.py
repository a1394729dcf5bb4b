"""Helpers for the GPU tests: moving numpy key arrays to/from CUDA tensors bit-for-bit, and
order checks on the device for the full-size property tests."""
import numpy as np

SIGNED_VIEW = {1: np.int8, 2: np.int16, 4: np.int32, 8: np.int64}


def to_dev(a: np.ndarray, offset_elems: int = 0):
    """Copy a to a CUDA tensor (int32/int64 view of the same bytes).  With offset_elems > 0
    the returned tensor starts that many elements into a larger allocation (unaligned when
    offset * itemsize is not a multiple of 16)."""
    import torch

    v = a.view(SIGNED_VIEW[a.dtype.itemsize])
    t = torch.from_numpy(v)
    if offset_elems:
        big = torch.empty(a.size + offset_elems, dtype=t.dtype, device="cuda")
        dev = big[offset_elems:]
        dev.copy_(t)
        return dev
    return t.cuda()


def from_dev(t, dtype) -> np.ndarray:
    return t.cpu().numpy().view(dtype)


def ordered_i64(t, dtype: str):
    """Device tensor of the reference order key as int64 comparable with signed compares."""
    import torch

    if dtype in ("u32", "i32", "f32"):
        u = t.view(torch.int32).to(torch.int64) & 0xFFFFFFFF
        if dtype == "i32":
            u = u ^ 0x80000000
        elif dtype == "f32":
            neg = (u & 0x80000000) != 0
            u = torch.where(neg, u ^ 0xFFFFFFFF, u ^ 0x80000000)
        return u  # in [0, 2^32)
    s = t.view(torch.int64)
    sign = torch.tensor(-(2 ** 63), dtype=torch.int64, device=t.device)
    if dtype == "u64":
        return s ^ sign  # unsigned order -> signed order
    if dtype == "i64":
        return s
    # f64: negative -> ~bits, positive -> bits ^ sign, then to signed order
    neg = s < 0
    o = torch.where(neg, ~s, s ^ sign)
    return o ^ sign


def is_sorted_dev(t, dtype: str) -> bool:
    o = ordered_i64(t, dtype)
    return bool((o[1:] >= o[:-1]).all().item())


def checksum_dev(t):
    """Order-independent checksum (sum and xor of 64-bit words) of a tensor's bytes."""
    import torch

    if t.element_size() == 4:
        w = t.view(torch.int32).to(torch.int64) & 0xFFFFFFFF
    else:
        w = t.view(torch.int64)
    s = int(w.sum().item())
    mixed = (w * 0x9E3779B1) ^ (w >> 7)
    return s, int(mixed.sum().item())
