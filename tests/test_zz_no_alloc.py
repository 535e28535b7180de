"""The allocation-free SSIM / MS-SSIM entry point (rg_ssim_plane_device_noalloc).

Some callers may not allocate device memory while they measure quality: their GPU memory is all
held by another allocator's pool, or their loop must not call cudaMalloc because it can stall the
whole device. This entry point keeps its working memory in a fixed array inside the library. The
test checks, through the C ABI, that two calls in a row on different plane pairs give the same
results as the allocating rg_ssim_plane and as the CPU oracle (within the 1e-6 tolerance of the
other SSIM tests) -- on a padded stride, on a plane too small for a second MS-SSIM scale (12x12) and
on a plane at the fixed limit (4096x510) -- that repeated calls leave the device's free memory
unchanged, and that planes beyond the fixed limit are refused with a clear error. It lives in its
own file, which pytest collects last, and passes alone in a fresh process as well as after the
other tests.
"""
import numpy as np
import pytest

from oracle_lib import ms_ssim_plane, ssim_plane as oracle_ssim

pytestmark = pytest.mark.gpu
TOL = 1e-6
# (width, height, row padding of the device planes)
SHAPES = [(1920, 1080, 0), (333, 197, 64), (12, 12, 0), (4096, 510, 0)]


def _pair(w, h, seed):
    rng = np.random.default_rng(seed)
    a = rng.integers(0, 256, (h, w), dtype=np.uint8)
    b = np.clip(a.astype(int) + rng.integers(-20, 21, (h, w)), 0, 255).astype(np.uint8)
    return a, b


def _device_plane(x, pad, dev):
    import torch
    h, w = x.shape
    t = torch.zeros((h, w + pad), dtype=torch.uint8, device=dev)
    t[:, :w] = torch.from_numpy(x).to(dev)
    return t


def test_noalloc_matches_allocating_entry_point_and_oracle_on_two_calls():
    import torch

    from ragdoll_b200.engine import ssim_plane, ssim_plane_device_noalloc

    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(device=dev)
    for seed, (w, h, pad) in enumerate(SHAPES):
        a, b = _pair(w, h, seed + 1)
        ta, tb = _device_plane(a, pad, dev), _device_plane(b, pad, dev)
        want = ssim_plane(a, b)
        ref = (oracle_ssim(a, b), ms_ssim_plane(a, b))
        for call in range(2):                       # two calls in a row share the fixed array
            out = torch.full((2,), -1.0, dtype=torch.float64, device=dev)
            torch.cuda.synchronize()
            ssim_plane_device_noalloc(ta.data_ptr(), w + pad, tb.data_ptr(), w + pad, w, h, out.data_ptr(),
                                      stream.cuda_stream)
            stream.synchronize()
            got = out.cpu().numpy()
            for k in range(2):
                assert abs(got[k] - want[k]) <= TOL, (w, h, pad, call, got, want)
                assert abs(got[k] - ref[k]) <= TOL, (w, h, pad, call, got, ref)


def test_noalloc_leaves_free_device_memory_unchanged():
    import torch

    from ragdoll_b200.engine import ssim_plane_device_noalloc

    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    a, b = _pair(1920, 1080, 7)
    ta, tb = _device_plane(a, 0, dev), _device_plane(b, 0, dev)
    out = torch.zeros(2, dtype=torch.float64, device=dev)
    ssim_plane_device_noalloc(ta.data_ptr(), 1920, tb.data_ptr(), 1920, 1920, 1080, out.data_ptr(), 0)  # warm-up
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(dev)
    for _ in range(3):
        ssim_plane_device_noalloc(ta.data_ptr(), 1920, tb.data_ptr(), 1920, 1920, 1080, out.data_ptr(), 0)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(dev)
    assert free1 == free0


def test_noalloc_rejects_planes_beyond_its_fixed_memory():
    import torch

    from ragdoll_b200.engine import RgError, ssim_plane_device_noalloc

    dev = torch.device("cuda:0")
    buf = torch.zeros(16, dtype=torch.uint8, device=dev)
    out = torch.zeros(2, dtype=torch.float64, device=dev)
    for w, h in [(3840, 2160), (4097, 8), (4, 64), (4096, 511)]:
        with pytest.raises(RgError) as e:
            ssim_plane_device_noalloc(buf.data_ptr(), w, buf.data_ptr(), w, w, h, out.data_ptr(), 0)
        assert e.value.code == -1
