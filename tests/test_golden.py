"""The oracle against the golden fixture made by the reference's own GPU kernels
(tests/golden/make_golden.py: k_packAB, cgemm_blk_t<false>, k_flush_cube,
k_diff, k_grid_cube, cuFFT from src/rx_host_corr.cu and src/cgemm.cuh).

Runs on the CPU: regenerates the same seeded packets, restates the path in the
oracle and compares bit for bit (packets, planes, per-channel visibilities),
and the FP64 image against the reference's FP32 image within 1e-4 of each
channel's peak (the reference grids with order-dependent float atomics).
"""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = os.path.join(HERE, "golden", "ref_v_update.json")


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.fixture(scope="module")
def golden():
    with open(FIXTURE) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def restated(golden):
    p = golden["params"]
    sky = oracle.sky_table(p["nant"], p["nch"], p["side_x"], p["sources"])
    pk = oracle.gen_packets(p["nant"], p["nch"], p["tpkt"], p["nheaps"], heap0=p["heap0"],
                            seq0=p["seq0"], port=p["udp_port"], sky=sky, sigma=p["sigma"],
                            seed=p["seed"])
    planes = oracle.corner_turn(pk, p["nant"], p["nch"], p["tpkt"], p["nheaps"])
    full = oracle.correlate(planes)
    return pk, planes, full


def test_packet_source_pinned(golden, restated):
    assert _sha(restated[0]) == golden["packets_sha256"]


def test_corner_turn_pinned_to_k_packAB(golden, restated):
    planes = restated[1]
    assert _sha(planes[0]) == golden["planes_re_sha256"]
    assert _sha(planes[1]) == golden["planes_im_sha256"]


def test_correlator_pinned_to_cgemm_blk_t(golden, restated):
    full = restated[2].astype("<i8")
    got = [_sha(full[c]) for c in range(full.shape[0])]
    assert got == golden["vis_sha256_per_channel"]
    for c, a, b, re, im in golden["vis_samples"]:
        assert (full[c, 0, a, b], full[c, 1, a, b]) == (re, im)


def test_image_pinned_to_reference_publish_path(golden, restated):
    p = golden["params"]
    img = oracle.image64(oracle.grid(restated[2], p["side_x"], p["grid"]))
    G = p["grid"]
    for c, ref in golden["images"].items():
        ref = np.asarray(ref, dtype=np.float64).reshape(G, G)
        scale = np.abs(ref).max()
        assert np.abs(img[int(c)] - ref).max() <= 1e-4 * scale
    vmax = img.reshape(img.shape[0], -1).max(1)
    ref_vmax = np.asarray(golden["image_vmax"])
    assert np.all(np.abs(vmax - ref_vmax) <= 1e-4 * np.abs(ref_vmax).max())
