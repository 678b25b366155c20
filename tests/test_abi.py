"""The C-ABI library loads and exports every function include/mixer.h declares;
argument validation happens before any device work (no GPU needed)."""
import ctypes as C
import os
import re

import pytest

import mixer

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    hdrs = [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))
            if f.endswith(".h")]
    names = set()
    for h in hdrs:
        text = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b(mixer_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_the_entry_points():
    names = _declared()
    assert "mixer_xcorr_tri" in names and "mixer_corner_turn" in names
    assert len(names) >= 25


@pytest.mark.parametrize("name", _declared())
def test_symbol_exported(name):
    lib = C.CDLL(mixer.LIB_PATH)
    assert hasattr(lib, name), f"{name} declared in include/ but not exported"


def test_python_binding_covers_header():
    assert set(_declared()) <= set(mixer.EXPORTED)


def test_layout_helpers():
    assert mixer.vis_tiles(256) == 3
    assert mixer.vis_tiles(1024) == 36
    assert mixer.vis_tiles(4096) == 528
    assert mixer.vis_tiles(96) == 1
    assert mixer.vis_elems(256, 128) == 128 * 3 * 2 * 128 * 128


def test_invalid_arguments_rejected_without_device_work():
    # bad shapes are refused before any CUDA call
    with pytest.raises(mixer.MixerError) as e:
        mixer.corner_turn(16, 8256, 64, 256, 128, 24, 8, 0, 16, 1024)   # tpkt % 16 != 0
    assert e.value.rc == mixer.EINVAL
    with pytest.raises(mixer.MixerError) as e:
        mixer.xcorr_tri(16, 256, 128, 1000, 0, 1000, mixer.VIS_ACC_I64, 16)  # kt % 16 != 0
    assert e.value.rc == mixer.EINVAL
    with pytest.raises(mixer.MixerError) as e:
        mixer.xcorr_tri(16, 256, 128, 131072, 0, 131072, mixer.VIS_ACC_I32, 16)
    assert e.value.rc == mixer.EOVERFLOW
    with pytest.raises(mixer.MixerError) as e:
        mixer.image_fft(16, 4, 48, 16)                                   # G not a power of 2
    assert e.value.rc == mixer.EINVAL


def test_desc_default_matches_wire():
    d = mixer.default_desc()
    assert (d.nant, d.nch, d.tpkt, d.pkt_stride, d.hdr_bytes) == (256, 128, 32, 8256, 64)
    assert d.ksub == 1024 and d.grid == 32 and d.side_x == 16
    assert mixer.WIRE_PAYLOAD_BYTES == 2 * d.nch * d.tpkt


def test_status_strings():
    lib = mixer.lib()
    for rc in (mixer.OK, mixer.EINVAL, mixer.ENOMEM, mixer.ETIMEOUT, mixer.EOVERFLOW):
        assert lib.mixer_strerror(rc)
