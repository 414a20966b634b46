"""Copies the VP8 decode fixtures the reference vendors (tests/fixtures/ of
oxideav-vp8: libvpx-encoded IVF streams with the libvpx-decoded I420
output, public conformance vectors) into tests/golden/vp8_fixtures/, so the
decoder restatement's tests run without the reference tree.

    python tests/golden/copy_vp8_fixtures.py <reference_root>

`reference_root` is the root of an oxideav-vp8 checkout (the directory that
holds its tests/fixtures/).
"""
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: copy_vp8_fixtures.py <reference_root>")
    src_root = os.path.join(sys.argv[1], "tests", "fixtures")
    dst_root = os.path.join(HERE, "vp8_fixtures")
    names = sorted(n for n in os.listdir(src_root) if os.path.isdir(os.path.join(src_root, n)))
    for name in names:
        os.makedirs(os.path.join(dst_root, name), exist_ok=True)
        for f in ("input.ivf", "expected.yuv"):
            shutil.copyfile(os.path.join(src_root, name, f), os.path.join(dst_root, name, f))
    print(f"copied {len(names)} fixtures into {dst_root}")


if __name__ == "__main__":
    main()
