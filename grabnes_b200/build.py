"""Build recipe of libgrabnes_gpu.so (sm_100a) -- compiled in-tree next to this file.

    python -m grabnes_b200.build            # or: python grabnes_b200/build.py

nvcc compiles every csrc/*.cu for sm_100a only; host code is compiled without FMA contraction so
that the host-side scalars of the neighbour search round as the reference's do.
"""
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libgrabnes_gpu.so")
OBJ = os.path.join(HERE, "_build")
DRIVER_DIR = os.path.join(HERE, "driver")
DRIVER = os.path.join(HERE, "grabnes")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-std=c++17", "-lineinfo", "--extended-lambda", "-Xcompiler", "-fPIC",
    "-Xcompiler", "-ffp-contract=off", "-Xptxas", "-O3",
]


def nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def build(verbose=False, jobs=8):
    os.makedirs(OBJ, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    hdrs = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(HERE, "..", "include", "*.h"))
    newest_hdr = max(os.path.getmtime(h) for h in hdrs)
    objs, procs = [], []
    for s in srcs:
        o = os.path.join(OBJ, os.path.basename(s)[:-3] + ".o")
        objs.append(o)
        if os.path.exists(o) and os.path.getmtime(o) >= max(os.path.getmtime(s), newest_hdr):
            continue
        cmd = [nvcc()] + NVCC_FLAGS + ["-c", s, "-o", o]
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((s, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
        while len([p for _, p in procs if p.poll() is None]) >= jobs:
            procs[0][1].wait()
    failed = []
    for s, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            failed.append((s, out))
        elif verbose and out.strip():
            print(out)
    if failed:
        raise RuntimeError("nvcc failed:\n" + "\n".join(f"--- {s}\n{o}" for s, o in failed))
    if not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", LIB] + objs + ["-lcudart"]
        subprocess.run(cmd, check=True)
    build_driver(verbose)
    return LIB


def build_driver(verbose=False):
    """The `grabnes Gendata.in` executable (host C++ over the C ABI), next to the library."""
    src = os.path.join(DRIVER_DIR, "grabnes.cpp")
    deps = [src, LIB] + glob.glob(os.path.join(HERE, "..", "include", "*.h")) + glob.glob(os.path.join(DRIVER_DIR, "*.inc"))
    if os.path.exists(DRIVER) and os.path.getmtime(DRIVER) >= max(os.path.getmtime(d) for d in deps):
        return DRIVER
    cxx = shutil.which("g++") or "g++"
    cmd = [cxx, "-O2", "-std=c++17", "-Wall", src, "-o", DRIVER, "-L" + HERE, "-lgrabnes_gpu",
           "-Wl,-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return DRIVER


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
