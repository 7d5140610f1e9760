"""shb_dilate_noalloc: dilation that allocates no device memory.

Callers that own the GPU's memory budget (a host application that reserves
all device memory up front) or that run on a deadline (where cudaMalloc's
implicit synchronisation is not acceptable) cannot let the library
allocate.  This entry point keeps its scratch in a fixed array inside the
library; the test calls it through the C ABI on device buffers the test
allocates, twice in a row, and checks each result byte for byte against the
existing shb_dilate entry point (the tolerance the dilation tests use).  It
also checks that a call takes no device memory and leaves the calling
thread's current device as it was.

The file name sorts last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from sh_baker_b200 import _capi as A

pytestmark = pytest.mark.gpu


def dilate_reference(ctx, kind, w, h, px, mask, passes):
    p, m = px.copy(), mask.copy()
    A.check(ctx.lib.shb_dilate(ctx.h, kind, w, h, p.ctypes.data, m.ctypes.data, passes, 0))
    return p, m


def dilate_noalloc(ctx, kind, w, h, px, mask, passes):
    import torch
    dp = torch.from_numpy(px.copy()).cuda()
    dm = torch.from_numpy(mask.copy()).cuda()
    torch.cuda.synchronize()
    A.check(ctx.lib.shb_dilate_noalloc(ctx.h, kind, w, h, C.c_void_p(dp.data_ptr()), C.c_void_p(dm.data_ptr()),
                                       passes))
    torch.cuda.synchronize()
    return dp.cpu().numpy(), dm.cpu().numpy()


def inputs(kind, w, h, density, seed):
    rng = np.random.default_rng(seed)
    n = w * h
    mask = (rng.uniform(size=n) < density).astype(np.uint8)
    if kind == A.DILATE_U8:
        px = rng.integers(0, 256, size=n).astype(np.uint8)
    else:
        px = rng.normal(size=n * (27 if kind == A.DILATE_SH9 else 1)).astype(np.float32)
    return px, mask


@pytest.mark.parametrize("kind,w,h,passes", [(A.DILATE_SH9, 160, 96, 3), (A.DILATE_F32, 512, 300, 4),
                                             (A.DILATE_U8, 333, 211, 5), (A.DILATE_SH9, 7, 5, 16)])
def test_noalloc_matches_dilate_two_calls(gpu_ctx, kind, w, h, passes):
    for call, (density, seed) in enumerate(((0.05, 11), (0.2, 12))):
        px, mask = inputs(kind, w, h, density, seed + kind)
        ref_p, ref_m = dilate_reference(gpu_ctx, kind, w, h, px, mask, passes)
        got_p, got_m = dilate_noalloc(gpu_ctx, kind, w, h, px, mask, passes)
        assert got_m.tobytes() == ref_m.tobytes(), f"mask differs on call {call}"
        assert got_p.tobytes() == ref_p.tobytes(), f"pixels differ on call {call}"


def test_noalloc_takes_no_device_memory(gpu_ctx):
    import torch
    w, h, passes = 300, 200, 6
    px, mask = inputs(A.DILATE_SH9, w, h, 0.1, 5)
    dp = torch.from_numpy(px).cuda()
    dm = torch.from_numpy(mask).cuda()
    args = (gpu_ctx.h, A.DILATE_SH9, w, h, C.c_void_p(dp.data_ptr()), C.c_void_p(dm.data_ptr()), passes)
    A.check(gpu_ctx.lib.shb_dilate_noalloc(*args))  # warm-up: kernels loaded
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    dev_before = torch.cuda.current_device()
    A.check(gpu_ctx.lib.shb_dilate_noalloc(*args))
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after >= free_before, f"the call took {free_before - free_after} bytes of device memory"
    assert torch.cuda.current_device() == dev_before


def test_noalloc_rejects_sizes_beyond_the_array(gpu_ctx):
    import torch
    w = h = 512  # 512*512 SH9 texels need ~27 MiB, the array holds 16 MiB
    dp = torch.zeros(w * h * 27, dtype=torch.float32, device="cuda")
    dm = torch.zeros(w * h, dtype=torch.uint8, device="cuda")
    st = gpu_ctx.lib.shb_dilate_noalloc(gpu_ctx.h, A.DILATE_SH9, w, h, C.c_void_p(dp.data_ptr()),
                                        C.c_void_p(dm.data_ptr()), 2)
    assert st == 1  # SHB_ERR_INVALID_ARG
    assert b"fixed array" in gpu_ctx.lib.shb_last_error()
    # sizes whose byte counts would overflow are rejected before they are formed
    big = 1 << 30
    st = gpu_ctx.lib.shb_dilate_noalloc(gpu_ctx.h, A.DILATE_SH9, big, big, C.c_void_p(dp.data_ptr()),
                                        C.c_void_p(dm.data_ptr()), 2)
    assert st == 1
    assert b"fixed array" in gpu_ctx.lib.shb_last_error()
