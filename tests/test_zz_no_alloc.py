"""mixer_image_noalloc: imaging with no device allocation.

Some callers cannot allocate device memory once they are running: a packet
capture framework that fixes every device buffer at start-up and treats a hidden
cudaMalloc as a budget violation, a real-time receive loop in which cudaMalloc or
cudaFree could stall or synchronise the GPU in the middle of a burst, or a host
process whose device allocator belongs to another runtime.  For them the
library keeps the gridding scratch in a fixed 16 MiB array of its own device
image instead of asking for a buffer.

These tests call that entry point through the C ABI twice in a row, on two
different visibility cubes, and check each image (and per-channel max / min)
  * against the FP64 oracle (exact int64 gridding of the oracle's V, then an
    FP64 FFT): max |img - img64| <= 1e-5 of the channel's peak, the image
    tolerance used throughout the suite;
  * against the allocating path (mixer_grid into a caller buffer, then
    mixer_image_fft) within the same tolerance.
The second call also shows the shared array was cleared between calls.  The
grids are 32, 64 and 128 cells wide, on arrays whose width (side_x) is not 16.
Requests the entry point must refuse (over its capacity, or a grid the FFT
cannot take) return MIXER_EINVAL and leave the shared array untouched.  The
file is named so pytest collects it last.
"""
import numpy as np
import pytest

import mixer
import oracle

pytestmark = pytest.mark.gpu

TOL = 1e-5     # of the channel's peak


def _full(nant, nch, seed):
    rng = np.random.default_rng(seed)
    planes = rng.integers(-90, 90, size=(2, nch, nant, 64), dtype=np.int8)
    return oracle.correlate(planes)


def _dev(cuda, arr):
    import torch
    return torch.from_numpy(np.ascontiguousarray(arr).reshape(-1)).to(cuda)


def _alloc_path(cuda, vis, nant, nch, side, G):
    import torch
    g = torch.zeros(nch * G * G * 2, dtype=torch.int64, device=cuda)
    img = torch.zeros(nch * G * G, dtype=torch.float32, device=cuda)
    vmax = torch.zeros(nch, dtype=torch.float32, device=cuda)
    vmin = torch.zeros(nch, dtype=torch.float32, device=cuda)
    mixer.grid(vis, nant, nch, side, G, g)
    mixer.image_fft(g, nch, G, img, vmax, vmin)
    return img, vmax, vmin


def _noalloc(cuda, vis, nant, nch, side, G):
    import torch
    img = torch.full((nch * G * G,), 7.0, dtype=torch.float32, device=cuda)
    vmax = torch.zeros(nch, dtype=torch.float32, device=cuda)
    vmin = torch.zeros(nch, dtype=torch.float32, device=cuda)
    mixer.image_noalloc(vis, nant, nch, side, G, img, vmax, vmin)
    return img, vmax, vmin


@pytest.mark.parametrize("nant,side,G,nch", [
    (240, 12, 32, 16),       # 12 x 20 array, 32 x 32 grid
    (300, 20, 64, 8),        # 20 x 15 array, 64 x 64 grid (three 128-row blocks)
    (512, 32, 128, 4),       # 32 x 16 array, 128 x 128 grid
])
def test_image_noalloc_matches_oracle_and_allocating_path(cuda, nant, side, G, nch):
    import torch
    for call, seed in enumerate((1, 2)):           # two calls in a row on the shared array
        full = _full(nant, nch, seed + 10 * G)
        img64 = oracle.image64(oracle.grid(full, side, G))                # [nch][G][G], FP64
        peak = np.abs(img64).max(axis=(1, 2))
        vis = _dev(cuda, oracle.vis_tile_pack(full))
        img, vmax, vmin = _noalloc(cuda, vis, nant, nch, side, G)
        ref_img, ref_max, ref_min = _alloc_path(cuda, vis, nant, nch, side, G)
        torch.cuda.synchronize()
        got = img.cpu().numpy().reshape(nch, G, G).astype(np.float64)
        err = np.abs(got - img64).max(axis=(1, 2))
        assert np.all(err <= TOL * peak), f"call {call}: error / peak {np.max(err / peak):.2e}"
        assert np.all(np.abs(vmax.cpu().numpy() - img64.max(axis=(1, 2))) <= TOL * peak)
        assert np.all(np.abs(vmin.cpu().numpy() - img64.min(axis=(1, 2))) <= TOL * peak)
        alloc = ref_img.cpu().numpy().reshape(nch, G, G)
        assert np.all(np.abs(got - alloc).max(axis=(1, 2)) <= TOL * peak), f"call {call}"
        assert np.all(np.abs(vmax.cpu().numpy() - ref_max.cpu().numpy()) <= TOL * peak)
        assert np.all(np.abs(vmin.cpu().numpy() - ref_min.cpu().numpy()) <= TOL * peak)


def test_image_noalloc_refuses_before_touching_the_array(cuda):
    """Oversize requests and grids the FFT cannot take are refused up front:
    an image made just before is still reproduced by an identical call after
    the refusals, and the refusals write nothing to their outputs."""
    import torch
    nant, side, G, nch = 256, 16, 32, 4
    full = _full(nant, nch, 7)
    vis = _dev(cuda, oracle.vis_tile_pack(full))
    first, _, _ = _noalloc(cuda, vis, nant, nch, side, G)
    torch.cuda.synchronize()
    out = torch.full((1 << 16,), 3.0, dtype=torch.float32, device=cuda)
    bad = [(nant, 65, side, 128),     # 65 * 128 * 128 > 2^20 cells
           (nant, 1, side, 256),      # the FFT takes G <= 128
           (nant, 1, side, 48),       # not a power of two
           (nant, 1, side, 2)]        # below the smallest FFT
    for n, c, s, g in bad:
        with pytest.raises(mixer.MixerError) as e:
            mixer.image_noalloc(vis, n, c, s, g, out)
        assert e.value.rc == mixer.EINVAL, (n, c, s, g)
    assert 65 * 128 * 128 > mixer.NOALLOC_MAX_CELLS
    again, _, _ = _noalloc(cuda, vis, nant, nch, side, G)
    torch.cuda.synchronize()
    assert torch.equal(first, again)
    assert bool((out == 3.0).all())
