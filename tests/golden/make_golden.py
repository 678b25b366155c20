"""Generate the golden fixture that pins the oracle to the reference's own GPU path.

Runs the reference's kernels -- k_packAB (src/rx_host_corr.cu:61-72),
cgemm_blk_t<false> (src/cgemm.cuh:28-69), k_flush_cube / k_diff / k_grid_cube
(:74-95) and its batched cuFFT plan (:205-206) -- compiled from the reference
sources into oracle/_ref/libref_gpu.so, on one V-update of the reference's
own shape (256 elements, 128 channels, 32 heaps x 32 samples = K 1024) of
seeded packets, and records:
  * sha256 of the packets (pins the packet source),
  * sha256 of the reference's A_re / A_im planes (pins the corner-turn),
  * per-channel sha256 of the reference's full-square V as little-endian int64
    [2][256][256] (pins the correlator, bit for bit),
  * the reference's live image (fftshifted real part) of three channels and the
    per-channel max (pins gridding + FFT to float tolerance).

Needs a B200 and the built oracle/_ref/libref_gpu.so.  Usage:
    python tests/golden/make_golden.py --out tests/golden/ref_v_update.json
"""
import argparse
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

PARAMS = {
    "nant": 256, "nch": 128, "tpkt": 32, "nheaps": 32, "side_x": 16, "grid": 32,
    "seed": 2024, "sigma": 16.0, "seq0": 0, "heap0": 0, "udp_port": 4096,
    # star A1 = 6 at (0.10, -0.05); planet A2 = 1.5 c / 128 at radius 0.2, orbit phase 0
    "sources": [[0.10, -0.05, 6.0, 0.0], [0.2, 0.0, 0.0, 1.5]],
    "image_channels": [0, 64, 127],
}


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def packets(p=PARAMS):
    import oracle
    sky = oracle.sky_table(p["nant"], p["nch"], p["side_x"], p["sources"])
    return oracle.gen_packets(p["nant"], p["nch"], p["tpkt"], p["nheaps"], heap0=p["heap0"],
                              seq0=p["seq0"], port=p["udp_port"], sky=sky, sigma=p["sigma"],
                              seed=p["seed"])


def main():
    import torch
    import oracle
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "ref_v_update.json"))
    args = ap.parse_args()
    p = PARAMS
    dev = torch.device("cuda:0")
    ref = oracle.ref_gpu()
    pk = packets()
    s = torch.cuda.current_stream().cuda_stream
    n, C, K = p["nant"], p["nch"], p["nheaps"] * p["tpkt"]
    bb = torch.from_numpy(pk.reshape(p["nheaps"] * n, -1)[:, 64:].copy()).to(dev)
    planes = [torch.zeros(C * n * K, dtype=torch.int8, device=dev) for _ in range(4)]
    cre = torch.zeros(C * n * n, dtype=torch.int32, device=dev)
    cim = torch.zeros_like(cre)
    assert ref.ref_pack(bb.data_ptr(), *[q.data_ptr() for q in planes], s) == 0
    assert ref.ref_cgemm(0, n, n, K, C, *[q.data_ptr() for q in planes], cre.data_ptr(),
                         cim.data_ptr(), s) == 0
    torch.cuda.synchronize()
    re = cre.cpu().numpy().reshape(C, n, n).astype("<i8")
    im = cim.cpu().numpy().reshape(C, n, n).astype("<i8")
    vis_sha = [sha(np.stack([re[c], im[c]])) for c in range(C)]
    # live-monitor path: flush -> diff -> grid -> FFT (:219-222), host shift (:233)
    vcube = torch.zeros(C * 2 * n * n, dtype=torch.float32, device=dev)
    vprev = torch.zeros_like(vcube)
    dv = torch.zeros_like(vcube)
    G = p["grid"]
    g = torch.zeros(C * G * G * 2, dtype=torch.float32, device=dev)
    im_c = torch.zeros_like(g)
    assert ref.ref_flush(vcube.data_ptr(), cre.data_ptr(), cim.data_ptr(), s) == 0
    assert ref.ref_diff(vcube.data_ptr(), vprev.data_ptr(), dv.data_ptr(), vcube.numel(), s) == 0
    assert ref.ref_grid(dv.data_ptr(), g.data_ptr(), s) == 0
    assert ref.ref_fft(g.data_ptr(), im_c.data_ptr(), s) == 0
    torch.cuda.synchronize()
    f = im_c.cpu().numpy().reshape(C, G, G, 2)[..., 0]
    img = np.roll(f, (-G // 2, -G // 2), axis=(1, 2))
    out = {
        "generator": "tests/golden/make_golden.py",
        "reference_kernels": ["k_packAB", "cgemm_blk_t<false>", "k_flush_cube", "k_diff",
                              "k_grid_cube", "cufftExecC2C"],
        "params": p,
        "packets_sha256": sha(pk),
        "planes_re_sha256": sha(planes[0].cpu().numpy()),
        "planes_im_sha256": sha(planes[1].cpu().numpy()),
        "vis_sha256_per_channel": vis_sha,
        "vis_samples": [[c, a, b, int(re[c, a, b]), int(im[c, a, b])]
                        for c, a, b in [(0, 0, 0), (5, 17, 3), (64, 255, 0), (127, 100, 200)]],
        "image_vmax": [float(v) for v in img.reshape(C, -1).max(1)],
        "image_vmin": [float(v) for v in img.reshape(C, -1).min(1)],
        "images": {str(c): img[c].ravel().tolist() for c in p["image_channels"]},
    }
    os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
    with open(args.out, "w") as fh:
        json.dump(out, fh)
    print(f"wrote {args.out}")


if __name__ == "__main__":
    main()
