"""Build recipe of the native parts of massccs_b200 (in-tree, sm_100a only).

    python -m massccs_b200.build          # libmassccs_gpu.so + the massccs CLI

Outputs:
    massccs_b200/lib/libmassccs_gpu.so    C-ABI engine (include/massccs_gpu.h)
    massccs_b200/lib/libmassccs_host.so   host set-up library (include/massccs_host.h)
    massccs_b200/bin/massccs              drop-in CLI (input.json -> report)
"""
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "lib")
BIN = os.path.join(PKG, "bin")
INC = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
              "--expt-relaxed-constexpr"]
HOST_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fopenmp", "-Wall", "-Wno-unused-variable"]


def _nvcc():
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newer(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build failed: " + " ".join(cmd[:3]) + " ...")
    return r


ENGINE_UNITS = ["ccs_engine.cu", "field.cu", "traj_field.cu", "setup_gpu.cu"]
ENGINE_HEADERS = ["ccs_device.cuh", "field_device.cuh", "engine_ctx.h"]


def build_engine(force=False, verbose=False):
    """libmassccs_gpu.so from its translation units, compiled in parallel."""
    from concurrent.futures import ThreadPoolExecutor
    os.makedirs(LIB, exist_ok=True)
    obj_dir = os.path.join(PKG, "_build")
    os.makedirs(obj_dir, exist_ok=True)
    out = os.path.join(LIB, "libmassccs_gpu.so")
    headers = [os.path.join(CSRC, f) for f in ENGINE_HEADERS] + [os.path.join(INC, "massccs_gpu.h")]
    objs, todo = [], []
    for u in ENGINE_UNITS:
        src = os.path.join(CSRC, u)
        obj = os.path.join(obj_dir, u.replace(".cu", ".o"))
        objs.append(obj)
        if force or _newer(obj, [src] + headers):
            cmd = [_nvcc()] + ARCH + NVCC_FLAGS + ["-c", "-o", obj, src]
            if verbose:
                cmd += ["-Xptxas", "-v"]
            todo.append(cmd)
    with ThreadPoolExecutor(max_workers=max(1, len(todo))) as ex:
        for r in ex.map(_run, todo):
            if verbose:
                sys.stderr.write(r.stderr)
    if force or todo or _newer(out, objs):
        _run([_nvcc()] + ARCH + ["-shared", "-o", out] + objs)
    return out


def build_host(force=False):
    """Host set-up library and the CLI (plain g++; they link the engine)."""
    os.makedirs(LIB, exist_ok=True)
    os.makedirs(BIN, exist_ok=True)
    hdir = os.path.join(CSRC, "host")
    if not os.path.isdir(hdir):
        return None
    cpp = sorted(os.path.join(hdir, f) for f in os.listdir(hdir) if f.endswith(".cpp") and f != "main.cpp")
    if not cpp:
        return None
    hdr = [os.path.join(hdir, f) for f in os.listdir(hdir) if f.endswith(".h")]
    lib_out = os.path.join(LIB, "libmassccs_host.so")
    deps = cpp + hdr + [os.path.join(INC, f) for f in os.listdir(INC)]
    gxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    engine = os.path.join(LIB, "libmassccs_gpu.so")
    if force or _newer(lib_out, deps + [engine]):
        _run([gxx] + HOST_FLAGS + ["-shared", "-I", INC, "-o", lib_out] + cpp +
             ["-L", LIB, "-lmassccs_gpu", "-Wl,-rpath,$ORIGIN"])
    main = os.path.join(hdir, "main.cpp")
    exe = os.path.join(BIN, "massccs")
    if os.path.exists(main) and (force or _newer(exe, deps + [main, lib_out])):
        _run([gxx] + HOST_FLAGS + ["-I", INC, "-o", exe, main,
                                   "-L", LIB, "-lmassccs_host", "-lmassccs_gpu",
                                   "-Wl,-rpath,$ORIGIN/../lib"])
    return lib_out


def build(force=False, verbose=False):
    build_engine(force=force, verbose=verbose)
    build_host(force=force)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print("built", LIB)
