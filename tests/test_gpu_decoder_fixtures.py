"""Parity against libvpx streams: the reference's decode fixtures
(tests/fixtures/*/input.ivf, produced by libvpx and decoded by it into
expected.yuv) are decoded by the oracle's decoder restatement — itself
pinned to expected.yuv byte for byte — with its capture hook on, and the
device kernels are fed each frame's captured state:

* vp8a_predict_inter_frame over the frame's decoded MB decisions and the
  references in force must equal the decoder's own §18 prediction of every
  inter MB (the prediction the reference's decoder forms in
  src/decoder.rs via predict_inter_mb / predict_split_mv,
  src/motion_comp.rs:1986, :2228), on the stream's filter set;
* vp8a_filter_frame over the frame's pre-filter reconstruction, its MBs'
  loop-filter records and the frame's filter configuration must equal the
  decoder's post-filter planes (src/loop_filter.rs:1364, :2506), for key
  and inter frames, normal and simple filters, segment and mode deltas.

Bit-exact on libvpx's own bitstreams, not only on synthetic decisions.
"""
import os

import numpy as np
import pytest

import vp8a
from vp8a import abi

pytestmark = pytest.mark.gpu

FIX = os.path.join(os.path.dirname(__file__), "golden", "vp8_fixtures")
NAMES = sorted(os.listdir(FIX)) if os.path.isdir(FIX) else []
REF_IDS = [abi.REF_LAST, abi.REF_GOLDEN, abi.REF_ALTREF]
# The fixtures that hold inter frames (the rest are single key frames).
WITH_INTER = {"altref-arnr-on", "golden-update-cycle", "i-frame-then-p-frame-64x64"}


@pytest.mark.parametrize("name", NAMES)
def test_device_kernels_on_libvpx_fixture(ctx, oracle, name):
    data = open(os.path.join(FIX, name, "input.ivf"), "rb").read()
    n_pred = n_lf = 0
    for i, f in enumerate(oracle.decode_ivf_captured(data)):
        if not f["key"]:
            inter = np.isin(f["dec"]["ref_frame"], REF_IDS)
            # Intra MBs keep the output's pixels: start from the capture's
            # zeros so the comparison covers the whole plane.
            out = tuple(np.zeros_like(p) for p in f["pred"])
            vp8a.predict_inter_frame(ctx, f["refs"], REF_IDS, f["dec"], out, full_pixel=f["version"] == 3,
                                     filter_set=vp8a.filter_set_for_version(f["version"]))
            for p, (g, w) in enumerate(zip(out, f["pred"])):
                bad = np.argwhere(g != w)
                assert bad.size == 0, f"frame {i} plane {p}: {len(bad)} px differ, first {bad[:3].tolist()}"
            n_pred += int(inter.sum())
        if f["filtered"]:
            got = vp8a.filter_frame(ctx, f["pre"], f["lf"], f["cfg"])
            for p, (g, w) in enumerate(zip(got, f["post"])):
                bad = np.argwhere(g != w)
                assert bad.size == 0, f"frame {i} plane {p}: {len(bad)} px differ after the loop filter"
            n_lf += 1
    assert (n_pred > 0) == (name in WITH_INTER)
