"""Build libg1cuda.so in-tree with nvcc for sm_100a (B200).

    python -m g1sim_b200.build [--force] [-v]    # or g1sim_b200.build.build()

Each translation unit under csrc/ (the plain step, the policy-fused
rollout, the adjoint, the surrogate) is compiled to an object in parallel,
then the objects are linked into one shared library written next to this
file (g1sim_b200/libg1cuda.so), so that it travels with the source tree;
nothing is installed anywhere else.  A unit is recompiled when it or a
header it includes (transitively) is newer than its object.
"""
import concurrent.futures as cf
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJDIR = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libg1cuda.so")
UNITS = ["g1_step.cu", "g1_step_k32.cu", "g1_step_k64.cu", "g1_step_k96.cu", "g1_step_k128.cu", "g1_step3_k64.cu",
         "g1_step3_k128.cu", "g1_policy.cu", "g1_adjoint.cu", "g1_surrogate.cu"]
SOURCES = [os.path.join(CSRC, u) for u in UNITS]
HEADERS = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))] + [
    os.path.join(os.path.dirname(HERE), "include", "g1sim_b200.h")]
DEPS = SOURCES + HEADERS

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++20", "-lineinfo"] + ARCH + ["-Xcompiler", "-fPIC"]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.sep not in c or os.path.exists(c)):
            return c
    return "nvcc"


def _obj(src):
    return os.path.join(OBJDIR, os.path.basename(src)[:-3] + ".o")


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def stale():
    return _newer(LIB, DEPS)


def _includes(path, seen=None):
    """Files under csrc/ and include/ that `path` includes, transitively."""
    seen = set() if seen is None else seen
    try:
        text = open(path).read()
    except OSError:
        return seen
    for name in re.findall(r'^\s*#\s*include\s+"([^"]+)"', text, re.M):
        dep = os.path.normpath(os.path.join(os.path.dirname(path), name))
        if dep not in seen and os.path.exists(dep):
            seen.add(dep)
            _includes(dep, seen)
    return seen


def _compile(src, verbose):
    obj = _obj(src)
    cmd = [nvcc()] + NVCC_FLAGS + (["-Xptxas", "-v"] if verbose else []) + ["-c", "-o", obj + ".tmp", src]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {os.path.basename(src)}:\n" + r.stdout + r.stderr)
    os.replace(obj + ".tmp", obj)
    return r.stdout + r.stderr


def build(force=False, verbose=False):
    if not force and not stale():
        return LIB
    os.makedirs(OBJDIR, exist_ok=True)
    todo = [s for s in SOURCES if force or _newer(_obj(s), [s] + sorted(_includes(s)))]
    with cf.ThreadPoolExecutor(max_workers=max(1, min(len(todo), os.cpu_count() or 1))) as ex:
        logs = list(ex.map(lambda s: _compile(s, verbose), todo))
    cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB + ".tmp"] + [_obj(s) for s in SOURCES]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc link failed:\n" + r.stdout + r.stderr)
    os.replace(LIB + ".tmp", LIB)
    if verbose:
        print("\n".join(logs))
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
