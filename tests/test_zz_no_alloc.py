"""mixer_image_noalloc: imaging with no device allocation.

Some callers cannot allocate device memory once they are running: a packet
capture framework that fixes every device buffer at start-up and treats a hidden
cudaMalloc as a budget violation, a real-time receive loop in which cudaMalloc or
cudaFree could stall or synchronise the GPU in the middle of a burst, or a host
process whose device allocator belongs to another runtime.  For them the
library keeps the gridding scratch in a fixed 16 MiB array of its own device
image instead of asking for a buffer.

This test calls that entry point through the C ABI twice in a row, on two
different visibility cubes, and checks each image (and per-channel max / min)
against the allocating path (mixer_grid into a caller buffer, then
mixer_image_fft) within the image tolerance used elsewhere in the suite:
max |difference| <= 1e-5 of the channel's peak.  The second call also shows the
shared array was cleared between calls.  Requests larger than the array are
refused with MIXER_EINVAL.  The file is named so pytest collects it last.
"""
import numpy as np
import pytest

import mixer
import oracle

pytestmark = pytest.mark.gpu


def _cube(cuda, nant, nch, seed):
    import torch
    rng = np.random.default_rng(seed)
    planes = rng.integers(-90, 90, size=(2, nch, nant, 64), dtype=np.int8)
    full = oracle.correlate(planes)
    return torch.from_numpy(oracle.vis_tile_pack(full).reshape(-1)).to(cuda)


def _alloc_path(cuda, vis, nant, nch, side, G):
    import torch
    g = torch.zeros(nch * G * G * 2, dtype=torch.int64, device=cuda)
    img = torch.zeros(nch * G * G, dtype=torch.float32, device=cuda)
    vmax = torch.zeros(nch, dtype=torch.float32, device=cuda)
    vmin = torch.zeros(nch, dtype=torch.float32, device=cuda)
    mixer.grid(vis, nant, nch, side, G, g)
    mixer.image_fft(g, nch, G, img, vmax, vmin)
    return img, vmax, vmin


def test_image_noalloc_matches_allocating_path(cuda):
    import torch
    nant, side, G, nch = 256, 16, 32, 16
    for call, seed in enumerate((1, 2)):
        vis = _cube(cuda, nant, nch, seed)
        img = torch.full((nch * G * G,), 7.0, dtype=torch.float32, device=cuda)
        vmax = torch.zeros(nch, dtype=torch.float32, device=cuda)
        vmin = torch.zeros(nch, dtype=torch.float32, device=cuda)
        mixer.image_noalloc(vis, nant, nch, side, G, img, vmax, vmin)
        ref_img, ref_max, ref_min = _alloc_path(cuda, vis, nant, nch, side, G)
        torch.cuda.synchronize()
        got = img.cpu().numpy().reshape(nch, -1)
        ref = ref_img.cpu().numpy().reshape(nch, -1)
        peak = np.abs(ref).max(axis=1, keepdims=True)
        assert np.all(np.abs(got - ref) <= 1e-5 * peak), f"call {call}"
        assert np.all(np.abs(vmax.cpu().numpy() - ref_max.cpu().numpy()) <= 1e-5 * peak[:, 0])
        assert np.all(np.abs(vmin.cpu().numpy() - ref_min.cpu().numpy()) <= 1e-5 * peak[:, 0])


def test_image_noalloc_refuses_oversize(cuda):
    import torch
    G, nch = 128, 65                                  # 65 * 128 * 128 > 2^20 cells
    assert nch * G * G > mixer.NOALLOC_MAX_CELLS
    vis = torch.zeros(16, dtype=torch.int64, device=cuda)
    img = torch.zeros(16, dtype=torch.float32, device=cuda)
    with pytest.raises(mixer.MixerError) as e:
        mixer.image_noalloc(vis, 256, nch, 16, G, img)
    assert e.value.rc == mixer.EINVAL
