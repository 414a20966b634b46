"""Build libvp8a.so in-tree for sm_100a.

    python oxideav-vp8_b200/vp8a/build.py [--force]

Compiles every csrc/*.cu (and the host-only csrc/*.cpp) with nvcc into vp8a/libvp8a.so. The library is built
with -fmad=false: the RD costs of the inter analysis are f64 expressions that
must round exactly like the reference's unfused arithmetic.
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(os.path.dirname(PKG), "include")
OUT = os.path.join(HERE, "libvp8a.so")

NVCC_FLAGS = [
    "-gencode",
    "arch=compute_100a,code=sm_100a",
    "-O3",
    "-lineinfo",
    "-fmad=false",
    "-std=c++17",
    "-Xcompiler",
    "-fPIC",
    "-shared",
]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def deps():
    return (sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) +
            glob.glob(os.path.join(INCLUDE, "*.h")))


def up_to_date():
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(p) <= t for p in deps())


def nvcc():
    for cand in ("nvcc", "/usr/local/cuda/bin/nvcc"):
        try:
            subprocess.run([cand, "--version"], check=True, capture_output=True)
            return cand
        except (OSError, subprocess.CalledProcessError):
            continue
    raise RuntimeError("nvcc not found")


def build(force=False, verbose=False):
    """Compiles each source to an object in parallel (objects under
    vp8a/_build/, rebuilt only when a source or header is newer), then links
    libvp8a.so."""
    if not force and up_to_date():
        return OUT
    import concurrent.futures as cf

    obj_dir = os.path.join(HERE, "_build")
    os.makedirs(obj_dir, exist_ok=True)
    compile_flags = [f for f in NVCC_FLAGS if f != "-shared"]
    headers = [p for p in deps() if p not in sources()]
    newest_header = max((os.path.getmtime(p) for p in headers), default=0.0)
    exe = nvcc()

    def compile_one(src):
        obj = os.path.join(obj_dir, os.path.basename(src) + ".o")
        if (not force and os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(src) and
                os.path.getmtime(obj) >= newest_header):
            return obj, None
        cmd = [exe] + compile_flags + ["-c", "-o", obj + ".tmp", src]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            return obj, r.stdout + r.stderr
        os.replace(obj + ".tmp", obj)
        return obj, None

    with cf.ThreadPoolExecutor(max_workers=max(1, min(len(sources()), os.cpu_count() or 1))) as ex:
        results = list(ex.map(compile_one, sources()))
    errors = [e for _, e in results if e]
    if errors:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errors))
    cmd = [exe] + NVCC_FLAGS + ["-o", OUT + ".tmp"] + [o for o, _ in results]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc link failed:\n" + r.stdout + r.stderr)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
