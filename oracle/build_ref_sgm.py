"""Build recipe: the reference's own SGM kernels as a library the tests can run (test infrastructure only).

    python oracle/build_ref_sgm.py <the reference's src directory>      -> oracle/_ref/libsgmref.so

The reference's dense SGM is CUDA source held in a Python string (src/xclean/stereo/sgm32.py, KERNELS) that it
compiles at run time with CuPy, which is not installed here.  This recipe reads that string out of the file (as text,
through the Python parser, without importing the module), writes it to oracle/_ref/sgm32_kernels.cu and compiles it
together with oracle/sgm_ref_host.cu (the launches the reference's SGM32.compute_gpu makes, restated in C++) into
oracle/_ref/libsgmref.so for sm_100a.  The library holds the reference's kernels unchanged; the GPU tests compare the
device SGM with it bit for bit.  oracle/_ref/ is not committed; it travels with the working tree to the GPU box.
"""
import ast
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUTDIR = os.path.join(HERE, "_ref")
OUT = os.path.join(OUTDIR, "libsgmref.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


def kernels_source(src_dir):
    path = os.path.join(src_dir, "xclean", "stereo", "sgm32.py")
    tree = ast.parse(open(path).read())
    for node in tree.body:
        if isinstance(node, ast.Assign) and any(getattr(t, "id", None) == "KERNELS" for t in node.targets):
            return node.value.value
    raise RuntimeError("KERNELS not found in %s" % path)


def build(src_dir):
    os.makedirs(OUTDIR, exist_ok=True)
    ku = os.path.join(OUTDIR, "sgm32_kernels.cu")
    with open(ku, "w") as fh:
        fh.write(kernels_source(src_dir))
    cmd = [NVCC, "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-Xcompiler", "-fPIC", "-shared",
           "-I", OUTDIR, os.path.join(HERE, "sgm_ref_host.cu"), "-o", OUT + ".tmp"]
    subprocess.check_call(cmd)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python %s <the reference's src directory>" % sys.argv[0])
    print(build(sys.argv[1]))
