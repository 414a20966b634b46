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
