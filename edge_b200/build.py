"""Builds ``edge_b200/libedge_b200.so`` in-tree with nvcc for sm_100a.

The library holds the host setup (host.cpp), the CUDA kernels and the C ABI declared in
``include/edge_b200.h``. Objects are compiled in parallel into ``edge_b200/_build`` and relinked only
when a source or header changed.

Usage: python -m edge_b200.build [-j N] [--force]
"""
import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libedge_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
                     "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _includes(path, seen=None):
    """The quoted #include files a source pulls in, transitively (searched beside the including
    file, in csrc and in include/), and the configuration list an inst_oN.cu names for its
    computed include (#define EDGE_B200_INC "...")."""
    seen = set() if seen is None else seen
    try:
        text = open(path).read()
    except OSError:
        return seen
    for line in text.splitlines():
        line = line.strip()
        if not (line.startswith("#include \"") or line.startswith("#define EDGE_B200_INC \"")):
            continue
        name = line.split('"')[1]
        for d in (os.path.dirname(path), CSRC, os.path.join(ROOT, "include")):
            cand = os.path.normpath(os.path.join(d, name))
            if os.path.exists(cand):
                if cand not in seen:
                    seen.add(cand)
                    _includes(cand, seen)
                break
    return seen


def _deps_mtime(src):
    return max([os.path.getmtime(h) for h in _includes(src)] + [0.0])


INST_PARTS = 4  # objects per order's kernel-set instantiations (kInstParts in inst_order.cuh)


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def units():
    """(source, part) per object: the order files inst_oN.cu once per part, the rest once."""
    out = []
    for s in sources():
        if os.path.basename(s).startswith("inst_o"):
            out += [(s, p) for p in range(INST_PARTS)]
        else:
            out.append((s, None))
    # the slowest objects first, so that they start before the short ones
    return sorted(out, key=lambda u: (u[1] is None, -int(os.path.basename(u[0])[6]) if u[1] is not None else 0))


def _compile(unit, force):
    src, part = unit
    hdr_mtime = _deps_mtime(src)
    obj = os.path.join(BUILD, os.path.basename(src) + (f".p{part}" if part is not None else "") + ".o")
    if (not force and os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(src)
            and os.path.getmtime(obj) >= hdr_mtime):
        return obj, False
    cmd = [nvcc()] + NVCC_FLAGS + (["-DEDGE_B200_PART=%d" % part] if part is not None else []) + ["-c", src, "-o", obj]
    if src.endswith(".cpp"):
        cmd = [nvcc(), "-x", "cu"] + NVCC_FLAGS + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj, True


def build(force=False, jobs=None, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    us = units()
    jobs = jobs or min(len(us), os.cpu_count() or 4)
    changed = False
    objs = []
    with cf.ThreadPoolExecutor(jobs) as ex:
        for obj, ch in ex.map(lambda u: _compile(u, force), us):
            objs.append(obj)
            changed |= ch
    if changed or force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart", "-lcuda"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
        if verbose:
            print("linked", LIB)
    build_probe(force=force)
    return LIB


PROBE_SRC = os.path.join(CSRC, "probe", "tc_probe.cu")
PROBE_LIB = os.path.join(HERE, "libedge_b200_probe.so")


def build_probe(force=False):
    """The tensor-core measurement probe (csrc/probe) as a library of its own."""
    if not force and os.path.exists(PROBE_LIB) and os.path.getmtime(PROBE_LIB) >= os.path.getmtime(PROBE_SRC):
        return PROBE_LIB
    cmd = [nvcc()] + NVCC_FLAGS + ["-shared", PROBE_SRC, "-o", PROBE_LIB]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {PROBE_SRC}:\n{r.stdout}\n{r.stderr}")
    return PROBE_LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, jobs=a.j, verbose=True))
