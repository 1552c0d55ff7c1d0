"""Build libnemo_b200.so in-tree: sm_100a kernels with nvcc, host code with g++.

    python -m nemo_b200.build          # incremental
    python -m nemo_b200.build --clean

Kernels: -gencode arch=compute_100a,code=sm_100a -lineinfo -O3 -fmad=false
(no FMA contraction, so float operation order matches the reference CPU
plugins). Host code: -O2 -ffp-contract=off (the glibc-matching candidate
functions are evaluated on the host when the correction tables are built and
must round exactly like the device).
"""

import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libnemo_b200.so")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")
CXX = shutil.which("g++") or "g++"   # not $CXX: it may point at a wrapper without OpenMP

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
INCLUDES = ["-I" + os.path.join(ROOT, "include"), "-I" + CSRC, "-I" + os.path.join(CUDA, "include")]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-prec-div=true", "-prec-sqrt=true",
                     "-ftz=false", "-Xcompiler", "-fPIC,-ffp-contract=off", "-ccbin", CXX] + INCLUDES
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-Wall", "-Wno-unused-parameter",
             "-pthread"] + INCLUDES
LINK = ["-shared", "-L" + os.path.join(CUDA, "lib64"), "-lcudart_static", "-lrt", "-ldl", "-lpthread",
        "-Wl,--exclude-libs,ALL"]


def _sources():
    cu = sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))
    cpp = sorted(f for f in os.listdir(CSRC) if f.endswith(".cpp"))
    return cu, cpp


def _headers_mtime():
    paths = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".hpp", ".cuh", ".h"))]
    paths += [os.path.join(ROOT, "include", f) for f in ("nemo.h", "nemo_b200.h")]
    paths += [os.path.join(ROOT, "include", "nemo", "types.h")]
    return max(os.path.getmtime(p) for p in paths if os.path.exists(p))


def _compile(src, verbose=False):
    path = os.path.join(CSRC, src)
    obj = os.path.join(BUILD, src + ".o")
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(path), _headers_mtime()):
        return obj
    if src.endswith(".cu"):
        cmd = [NVCC] + NVCC_FLAGS + ["-c", path, "-o", obj]
    else:
        cmd = [CXX] + CXX_FLAGS + ["-c", path, "-o", obj]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("compiling %s failed:\n%s%s" % (src, r.stdout, r.stderr))
    return obj


def build(verbose=False, clean=False):
    if clean and os.path.isdir(BUILD):
        shutil.rmtree(BUILD)
    os.makedirs(BUILD, exist_ok=True)
    cu, cpp = _sources()
    with concurrent.futures.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), cu + cpp))
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(o) for o in objs):
        return LIB
    tmp = LIB + ".tmp"
    cmd = [CXX] + objs + LINK + ["-o", tmp]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("linking failed:\n%s%s" % (r.stdout, r.stderr))
    os.replace(tmp, LIB)
    return LIB


def build_plugin(src, name=None, plugin_dir=None, extra_flags=()):
    """Compile a GPU neuron-model plugin (include/nemo_b200_plugin.h) from the
    CUDA source `src` into <plugin_dir>/b200/lib<name>.so, the place the
    library looks for it beside <name>.ini (name: the source's base name;
    plugin_dir: the source's directory). Rebuilt only when the source or the
    plugin header is newer. Returns the library's path."""
    name = name or os.path.splitext(os.path.basename(src))[0]
    plugin_dir = plugin_dir or os.path.dirname(os.path.abspath(src))
    out = os.path.join(plugin_dir, "b200", "lib%s.so" % name)
    header = os.path.join(ROOT, "include", "nemo_b200_plugin.h")
    if os.path.exists(out) and os.path.getmtime(out) >= max(os.path.getmtime(src), os.path.getmtime(header)):
        return out
    os.makedirs(os.path.dirname(out), exist_ok=True)
    cmd = [NVCC] + ARCH + ["-O3", "-lineinfo", "-fmad=false", "-shared", "-Xcompiler", "-fPIC", "-ccbin", CXX,
                           "-I" + os.path.join(ROOT, "include"), "-Xlinker", "--exclude-libs,ALL",
                           *extra_flags, src, "-o", out + ".tmp"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("building plugin %s failed:\n%s%s" % (src, r.stdout, r.stderr))
    os.replace(out + ".tmp", out)
    return out


def prepare_tables():
    """Write the glibc correction-table cache next to the library."""
    import ctypes
    dll = ctypes.CDLL(LIB)
    dll.nemo_strerror.restype = ctypes.c_char_p
    if dll.nemo_b200_prepare_libm_tables() != 0:
        raise RuntimeError(dll.nemo_strerror().decode())


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, clean="--clean" in sys.argv)
    prepare_tables()
    print(LIB)
