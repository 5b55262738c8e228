"""Build libxcb200.so (sm_100a) in-tree with nvcc.

Frontend sources are compiled with --fmad=false and IEEE division / square root: their results must match the
reference bit for bit, and every fused multiply-add there is an explicit intrinsic.  The bundle-adjustment sources may
contract (their parity is a stated tolerance)."""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INC = os.path.join(os.path.dirname(HERE), "include")
OUT = os.path.join(HERE, "libxcb200.so")
BUILD = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I", CSRC, "-I", INC] + ARCH
STRICT = ["--fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false"]

SOURCES = {
    "front_detect.cu": STRICT,
    "front_orb_match.cu": STRICT,
    "front_stereo.cu": STRICT,
    "front_api.cu": STRICT,
    "front_mapmatch.cu": STRICT,
    "ba_posefree.cu": STRICT,
    "stereo_sgm.cu": STRICT,
    "front_ext.cu": STRICT,
    "ba_window.cu": [],
    "ba_api.cu": [],
}


def _sources():
    srcs = dict(SOURCES)
    for fn in sorted(os.listdir(CSRC)):
        if fn.endswith(".cu") and fn not in srcs:
            srcs[fn] = []
    return srcs


def _newer(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, extra=()):
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers += [os.path.join(INC, f) for f in os.listdir(INC)]
    srcs = _sources()
    objs = []
    jobs = []
    for fn, flags in srcs.items():
        src = os.path.join(CSRC, fn)
        obj = os.path.join(BUILD, fn.replace(".cu", ".o"))
        objs.append(obj)
        if force or _newer(obj, [src] + headers):
            jobs.append([NVCC] + COMMON + list(flags) + list(extra) + ["-c", src, "-o", obj])

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed:\n%s\n%s" % (" ".join(cmd), r.stderr))
        if verbose and r.stderr.strip():
            print(r.stderr)
        return r

    with ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        list(ex.map(run, jobs))
    if force or jobs or _newer(OUT, objs):
        tmp = OUT + ".tmp"
        run([NVCC] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcuda"])
        os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    extra = []
    if "--ptxas-v" in sys.argv:
        extra = ["-Xptxas", "-v"]
    print(build(force="--force" in sys.argv or bool(extra), verbose="-v" in sys.argv or bool(extra), extra=extra))
