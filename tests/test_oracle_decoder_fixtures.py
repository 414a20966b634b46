"""Pins the oracle's decoder restatement (oracle/decoder.c) — and through it
the restated §14 inverse transforms, §18 inter prediction and §15 loop
filter it reuses — to the libvpx-produced decode fixtures the reference
vendors (tests/fixtures/, copied into tests/golden/vp8_fixtures/ by
tests/golden/copy_vp8_fixtures.py). Each stream's decoded pictures,
concatenated, must equal expected.yuv byte for byte; like the reference's
own fixture tests (src/state.rs:1937-2030, src/decoder.rs tests), a stream
whose expected file holds fewer pictures than it decodes is compared on the
expected prefix.
"""
import os

import numpy as np
import oracle
import pytest

FIX = os.path.join(os.path.dirname(__file__), "golden", "vp8_fixtures")
NAMES = sorted(os.listdir(FIX)) if os.path.isdir(FIX) else []


@pytest.fixture(autouse=True, scope="module")
def _oracle_built(request):
    request.getfixturevalue("oracle")


@pytest.mark.parametrize("name", NAMES)
def test_decoder_matches_libvpx_fixture(name):
    data = open(os.path.join(FIX, name, "input.ivf"), "rb").read()
    expected = np.fromfile(os.path.join(FIX, name, "expected.yuv"), np.uint8)
    got = np.concatenate([np.concatenate([p.reshape(-1) for p in pic]) for pic, _ in oracle.decode_ivf(data)])
    assert got.size >= expected.size, (got.size, expected.size)
    got = got[:expected.size]
    bad = np.flatnonzero(got != expected)
    assert bad.size == 0, f"{bad.size} bytes differ, first at {bad[:8]}"


def test_all_fixtures_present():
    assert len(NAMES) == 13


def _planes_equal(a, b):
    return all(np.array_equal(x, y) for x, y in zip(a, b))


@pytest.mark.parametrize("name", ["i-frame-then-p-frame-64x64", "golden-update-cycle", "altref-arnr-on",
                                  "vp8-with-loopfilter-mode-simple"])
def test_decoder_capture_is_consistent(name):
    # The capture hook's intermediate state re-derives the decoded pictures:
    # the batched prediction entry point over the captured decisions
    # reproduces the decoder's own per-MB prediction, the frame filter over
    # the captured records reproduces the post-filter planes, and those crop
    # to the visible picture. This is the state the device parity test
    # feeds to the CUDA kernels.
    from vp8a import abi
    from vp8a.api import filter_set_for_version

    data = open(os.path.join(FIX, name, "input.ivf"), "rb").read()
    n_inter = 0
    for f in oracle.decode_ivf_captured(data):
        if not f["key"]:
            n_inter += 1
            inter = np.isin(f["dec"]["ref_frame"], [abi.REF_LAST, abi.REF_GOLDEN, abi.REF_ALTREF])
            assert inter.any()
            out = tuple(np.zeros_like(p) for p in f["pred"])
            oracle.predict_inter_frame(f["refs"], [abi.REF_LAST, abi.REF_GOLDEN, abi.REF_ALTREF], f["dec"], out,
                                       full_pixel=f["version"] == 3, filter_set=filter_set_for_version(f["version"]))
            assert _planes_equal(out, f["pred"])
        post = oracle.filter_frame(f["pre"], f["lf"], f["cfg"]) if f["filtered"] else f["pre"]
        assert _planes_equal(post, f["post"])
        y, u, v = f["picture"]
        assert np.array_equal(f["post"][0][:y.shape[0], :y.shape[1]], y)
        assert np.array_equal(f["post"][1][:u.shape[0], :u.shape[1]], u)
    assert n_inter > 0 or name == "vp8-with-loopfilter-mode-simple"  # a single key frame
