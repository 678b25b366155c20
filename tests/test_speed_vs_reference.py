"""Speed of the X-engine's tensor-core triangle cGEMM against the reference's own
wmma kernel (cgemm_blk_t<true>, src/cgemm.cuh:28-69) compiled from its sources
for sm_100a, on the same B200 and the same int8 inputs: one V-update of the
larger plain array (N 1024, C 256, K 1024).  Prints both times; the
X-engine must be faster.  Run with -s to see the numbers."""
import numpy as np
import pytest

import mixer
import oracle

pytestmark = pytest.mark.gpu


def _time(fn, reps=5):
    import torch
    fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def test_faster_than_reference_wmma(cuda):
    import torch
    if not oracle.ref_gpu_available():
        pytest.skip("oracle/_ref/libref_gpu.so not built")
    ref = oracle.ref_gpu()
    N, C, K = 1024, 256, 1024
    g = torch.Generator(device=cuda).manual_seed(5)
    xr = torch.randint(-127, 128, (C * N * K,), dtype=torch.int8, device=cuda, generator=g)
    xi = torch.randint(-127, 128, (C * N * K,), dtype=torch.int8, device=cuda, generator=g)
    nxi = -xi                                   # the reference's B_im = -X_im plane
    cre = torch.zeros(C * N * N, dtype=torch.int32, device=cuda)
    cim = torch.zeros_like(cre)
    s = torch.cuda.current_stream().cuda_stream
    t_ref = _time(lambda: ref.ref_cgemm(1, N, N, K, C, xr.data_ptr(), xi.data_ptr(), xr.data_ptr(),
                                        nxi.data_ptr(), cre.data_ptr(), cim.data_ptr(), s))
    planes = torch.cat([xr, xi])
    vis = torch.zeros(mixer.vis_elems(N, C), dtype=torch.int64, device=cuda)
    t_ours = _time(lambda: mixer.xcorr_tri(planes, N, C, K, 0, K, mixer.VIS_ACC_I64, vis))
    ops = 8.0 * N * (N + 1) / 2 * K * C
    print(f"\nreference cgemm_blk_t<true> (full square, int32 RMW): {t_ref:.3f} ms "
          f"= {ops / t_ref / 1e9:.0f} TOPS triangle-basis")
    print(f"X-engine k_xcorr_tri (lower triangle, int64 RMW):    {t_ours:.3f} ms "
          f"= {ops / t_ours / 1e9:.0f} TOPS triangle-basis; speed-up {t_ref / t_ours:.1f}x")
    # same numbers: lower triangle of the reference's cube equals ours
    cre.zero_(); cim.zero_(); vis.zero_()
    ref.ref_cgemm(0, N, N, K, 4, xr.data_ptr(), xi.data_ptr(), xr.data_ptr(), nxi.data_ptr(),
                  cre.data_ptr(), cim.data_ptr(), s)
    mixer.xcorr_tri(planes, N, C, K, 0, K, mixer.VIS_ACC_I64, vis)
    full = torch.zeros(C * 2 * N * N, dtype=torch.int64, device=cuda)
    mixer.vis_unpack_i64(vis, N, C, full)
    torch.cuda.synchronize()
    full = full.view(C, 2, N, N)[:4]
    assert torch.equal(full[:, 0], cre.view(-1, N, N)[:4].to(torch.int64))
    assert torch.equal(full[:, 1], cim.view(-1, N, N)[:4].to(torch.int64))
    assert t_ours < t_ref
