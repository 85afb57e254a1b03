"""Build the engine's shared library, libacp_cuda.so, in-tree for sm_100a.

nvcc compiles the CUDA kernels and the C ABI (csrc/*.cu, csrc/*.cpp) into
acpulse_vclbm_b200/libacp_cuda.so; no torch extension machinery is involved.
Runs without a GPU (cross-compilation).

usage: python -m acpulse_vclbm_b200.build [--force] [--verbose-ptxas]
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libacp_cuda.so")
MAIN = os.path.join(HERE, "acp_main")
HOSTCXX = os.environ.get("ACP_HOSTCXX", "/usr/bin/g++")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["engine.cu", "batch.cu", "caseparse.cpp"]


def _deps():
    files = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    files.append(os.path.join(os.path.dirname(HERE), "include", "acp.h"))
    files.append(os.path.abspath(__file__))
    return files


def up_to_date():
    if not os.path.exists(OUT) or not os.path.exists(MAIN):
        return False
    t = min(os.path.getmtime(OUT), os.path.getmtime(MAIN))
    host = [os.path.join(HERE, "host", f) for f in os.listdir(os.path.join(HERE, "host"))]
    return all(os.path.getmtime(f) <= t for f in _deps() + host)


def build_host():
    """The drop-in C++ Control/Lattice and the reference-style driver, linked to libacp_cuda.so."""
    host = os.path.join(HERE, "host")
    srcs = [os.path.join(host, f) for f in ("Control.cpp", "Lattice.cpp", "Node.cpp", "acp_main.cpp")]
    subprocess.run([HOSTCXX, "-O2", "-std=c++17", "-o", MAIN, *srcs, "-L" + HERE, "-lacp_cuda",
                    "-Wl,-rpath,$ORIGIN"], check=True)
    return MAIN


def build(force=False, verbose_ptxas=False):
    if not force and up_to_date():
        return OUT
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs, cmds = [], []
    for src in SOURCES:
        obj = os.path.join(objdir, src + ".o")
        cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
               "--expt-relaxed-constexpr", "-c", os.path.join(CSRC, src), "-o", obj]
        if src.endswith(".cpp"):
            cmd.insert(1, "-x")
            cmd.insert(2, "cu")
        if verbose_ptxas:
            cmd += ["-Xptxas", "-v"]
        cmds.append(cmd)
        objs.append(obj)
    # the translation units compile side by side
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(len(cmds)) as pool:
        for r in pool.map(lambda c: subprocess.run(c, capture_output=True, text=True), cmds):
            if r.returncode != 0:
                sys.stderr.write(r.stdout + r.stderr)
                raise subprocess.CalledProcessError(r.returncode, r.args)
            if verbose_ptxas:
                sys.stderr.write(r.stderr)
    tmp = OUT + ".tmp"
    subprocess.run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", tmp, *objs], check=True)
    os.replace(tmp, OUT)
    build_host()
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose_ptxas="--verbose-ptxas" in sys.argv)
    print(OUT)
