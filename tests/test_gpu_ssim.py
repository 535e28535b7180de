"""SSIM / MS-SSIM / PSNR / VMAF-Lite on the GPU against the oracle (GPU tests).

Tolerance: 1e-6 absolute for SSIM and MS-SSIM (the reference's per-row f32 order is reproduced,
so the plane SSIM agrees to the last bit in practice; MS-SSIM's final pow runs in f64 on the
host), 1e-9 for PSNR (integer SSE), 1e-9 on the 0..100 VMAF-Lite score (its f64 block terms are
summed per block row, then row by row, instead of in one raster-order sum), 1e-4 dB for SSIM in dB
(-10 log10(1 - SSIM) amplifies SSIM's tolerance near 1).
"""
import numpy as np
import pytest

import oracle_lib
from ragdoll_b200.synth import grating_clip, synth_video_frame

pytestmark = pytest.mark.gpu
TOL = 1e-6


@pytest.mark.parametrize("w,h", [(1920, 1080), (333, 197), (64, 36), (9, 9), (15, 33)])
def test_ssim_plane_matches_oracle(w, h):
    from ragdoll_b200.engine import ssim_plane
    rng = np.random.default_rng(w * 31 + h)
    a = rng.integers(0, 256, (h, w), dtype=np.uint8)
    b = np.clip(a.astype(int) + rng.integers(-12, 13, (h, w)), 0, 255).astype(np.uint8)
    s, m = ssim_plane(a, b)
    assert abs(s - oracle_lib.ssim_plane(a, b)) <= TOL
    assert abs(m - oracle_lib.ms_ssim_plane(a, b)) <= TOL


def test_ssim_identical_planes_is_one():
    from ragdoll_b200.engine import ssim_plane
    a = synth_video_frame(160, 90, 3)[0]
    s, m = ssim_plane(a, a)
    assert s == pytest.approx(1.0, abs=1e-7) and m == pytest.approx(1.0, abs=1e-7)


def test_quality_of_reconstruction_matches_oracle():
    """rg_quality_frame on the engine's reconstruction equals the oracle's metrics of the
    oracle's (identical) reconstruction: Y/U/V SSIM, the 4:1:1 average, MS-SSIM, PSNR."""
    from ragdoll_b200.engine import RG_FRAME_IDR, RG_FRAME_P, RG_PROFILE_HIGH, Engine
    w, h, qp = 352, 288, 30
    frames = grating_clip(w, h, 3, seed=5, motion=5.0, rects=2)
    eng = Engine(w, h, qp, profile=RG_PROFILE_HIGH)
    for i, fr in enumerate(frames):
        eng.analyse([fr], [RG_FRAME_IDR if i == 0 else RG_FRAME_P])
        q = eng.quality(fr)
        ry, ru, rv = eng.recon()
        assert abs(q["ssim_y"] - oracle_lib.ssim_plane(fr[0], ry)) <= TOL
        assert abs(q["ssim_u"] - oracle_lib.ssim_plane(fr[1], ru)) <= TOL
        assert abs(q["ssim_v"] - oracle_lib.ssim_plane(fr[2], rv)) <= TOL
        assert abs(q["ms_ssim"] - oracle_lib.ms_ssim_plane(fr[0], ry)) <= TOL
        assert abs(q["ssim_avg"] - (4 * q["ssim_y"] + q["ssim_u"] + q["ssim_v"]) / 6) <= 1e-12
        assert q["psnr_y"] == pytest.approx(oracle_lib.psnr_plane(fr[0], ry), abs=1e-9)
        assert q["psnr_u"] == pytest.approx(oracle_lib.psnr_plane(fr[1], ru), abs=1e-9)
        assert q["psnr_v"] == pytest.approx(oracle_lib.psnr_plane(fr[2], rv), abs=1e-9)


VMAF_TOL = 1e-9  # f64 sums per block row then in row order vs one raster-order sum: rounding only


@pytest.mark.parametrize("w,h", [(1920, 1080), (333, 197), (64, 36), (7, 9), (3, 40)])
@pytest.mark.parametrize("with_prev", [False, True])
def test_vmaf_lite_plane_matches_oracle(w, h, with_prev):
    from ragdoll_b200.engine import vmaf_lite_plane
    rng = np.random.default_rng(w * 7 + h)
    a = rng.integers(0, 256, (h, w), dtype=np.uint8)
    b = np.clip(a.astype(int) + rng.integers(-20, 21, (h, w)), 0, 255).astype(np.uint8)
    prev = np.roll(a, 3, axis=1) if with_prev else None
    got = vmaf_lite_plane(a, b, prev)
    assert abs(got - oracle_lib.vmaf_lite_plane(a, b, prev)) <= VMAF_TOL
    assert vmaf_lite_plane(a, a) == 100.0


def test_quality_report_of_reconstruction_matches_oracle():
    """The whole evaluate_frame_quality report of the engine's reconstruction, with the previous
    source frame for VMAF-Lite's motion term, against the oracle's report."""
    import math
    from ragdoll_b200.engine import RG_FRAME_IDR, RG_FRAME_P, RG_PROFILE_MAIN, Engine
    w, h, qp = 320, 180, 34
    frames = grating_clip(w, h, 3, seed=8, motion=6.0, rects=2)
    eng = Engine(w, h, qp, profile=RG_PROFILE_MAIN)
    for i, fr in enumerate(frames):
        eng.analyse([fr], [RG_FRAME_IDR if i == 0 else RG_FRAME_P])
        prev = frames[i - 1] if i else None
        q = eng.quality(fr, prev=prev)
        want = oracle_lib.quality_report(fr, eng.recon(), prev)
        for key in ("psnr_y", "psnr_u", "psnr_v", "psnr_avg", "psnr_yuv_611"):
            assert q[key] == pytest.approx(want[key], abs=1e-9), key
        for key in ("ssim_y", "ssim_u", "ssim_v", "ssim_avg", "ms_ssim"):
            assert abs(q[key] - want[key]) <= TOL, key
        assert abs(q["ssim_db"] - want["ssim_db"]) <= 1e-4 and math.isfinite(q["ssim_db"])
        assert abs(q["vmaf_lite"] - want["vmaf_lite"]) <= VMAF_TOL


def test_batched_ssim_of_many_pairs_matches_oracle():
    """rg_ssim_batch_device: every pair of a batch (device planes, padded stride) equals the
    oracle's SSIM and MS-SSIM within 1e-6, in one set of shared launches."""
    import torch

    from oracle_lib import ms_ssim_plane
    from oracle_lib import ssim_plane as oracle_ssim
    from ragdoll_b200.engine import ssim_batch_device
    w, h, pad, n = 333, 197, 32, 6
    rng = np.random.default_rng(9)
    a = rng.integers(0, 256, (n, h, w)).astype(np.uint8)
    b = np.clip(a.astype(int) + rng.integers(-25, 26, (n, h, w)), 0, 255).astype(np.uint8)
    da = torch.zeros((n, h, w + pad), dtype=torch.uint8, device="cuda")
    db = torch.zeros((n, h, w + pad), dtype=torch.uint8, device="cuda")
    da[:, :, :w] = torch.from_numpy(a).cuda()
    db[:, :, :w] = torch.from_numpy(b).cuda()
    s, m = ssim_batch_device([da[i].data_ptr() for i in range(n)], [db[i].data_ptr() for i in range(n)], w, h,
                             w + pad, w + pad)
    for i in range(n):
        assert abs(s[i] - oracle_ssim(a[i], b[i])) <= 1e-6
        assert abs(m[i] - ms_ssim_plane(a[i], b[i])) <= 1e-6
