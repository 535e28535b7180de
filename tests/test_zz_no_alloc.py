"""The allocation-free SSIM / MS-SSIM entry point (rg_ssim_plane_device_noalloc).

Some callers may not allocate device memory while they measure quality: their GPU memory is all
held by another allocator's pool, or their loop must not call cudaMalloc because it can stall the
whole device. This entry point keeps its working memory in a fixed array inside the library. The
test checks, through the C ABI, that two calls in a row on different plane pairs give the same
results as the allocating rg_ssim_plane (within the 1e-6 tolerance of the other SSIM tests), and
that planes beyond the fixed limit are refused with a clear error. It lives in its own file, which
pytest collects last, and passes alone in a fresh process as well as after the other tests.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-6


def _pair(w, h, seed):
    rng = np.random.default_rng(seed)
    a = rng.integers(0, 256, (h, w), dtype=np.uint8)
    b = np.clip(a.astype(int) + rng.integers(-20, 21, (h, w)), 0, 255).astype(np.uint8)
    return a, b


def test_noalloc_matches_allocating_entry_point_on_two_calls():
    import torch

    from ragdoll_b200.engine import ssim_plane, ssim_plane_device_noalloc

    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(device=dev)
    for seed, (w, h) in enumerate([(1920, 1080), (333, 197)]):
        a, b = _pair(w, h, seed + 1)
        ta, tb = torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)
        out = torch.full((2,), -1.0, dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        ssim_plane_device_noalloc(ta.data_ptr(), w, tb.data_ptr(), w, w, h, out.data_ptr(), stream.cuda_stream)
        stream.synchronize()
        got = out.cpu().numpy()
        want = ssim_plane(a, b)
        assert abs(got[0] - want[0]) <= TOL, (w, h, got, want)
        assert abs(got[1] - want[1]) <= TOL, (w, h, got, want)


def test_noalloc_rejects_planes_beyond_its_fixed_memory():
    import torch

    from ragdoll_b200.engine import RgError, ssim_plane_device_noalloc

    dev = torch.device("cuda:0")
    buf = torch.zeros(16, dtype=torch.uint8, device=dev)
    out = torch.zeros(2, dtype=torch.float64, device=dev)
    for w, h in [(3840, 2160), (4097, 8), (4, 64)]:
        with pytest.raises(RgError) as e:
            ssim_plane_device_noalloc(buf.data_ptr(), w, buf.data_ptr(), w, w, h, out.data_ptr(), 0)
        assert e.value.code == -1
