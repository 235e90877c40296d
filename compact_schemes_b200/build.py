"""Build libcompact_b200.so in-tree for sm_100a (nvcc cross-compiles; no GPU needed).

    python -m compact_schemes_b200.build      # or: python compact_schemes_b200/build.py
"""
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libcompact_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
         "-Xcompiler", "-ffp-contract=off",
         "--expt-relaxed-constexpr", "-I" + os.path.join(os.path.dirname(HERE), "include")]


def sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def _headers_mtime():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(os.path.dirname(HERE), "include", "compact_b200.h"))
    return max(os.path.getmtime(h) for h in hs)


def _compile(src, verbose_regs=False):
    obj = os.path.join(BUILD, src + ".o")
    path = os.path.join(CSRC, src)
    if (os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(path)
            and os.path.getmtime(obj) >= _headers_mtime() and not verbose_regs):
        return obj, ""
    cmd = [NVCC, *ARCH, *FLAGS, "-c", "-o", obj]
    if src.endswith(".cpp"):
        cmd += ["-x", "cu"]
    if verbose_regs:
        cmd += ["-Xptxas", "-v"]
    cmd.append(path)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode:
        raise RuntimeError("nvcc failed for %s:\n%s%s" % (src, r.stdout, r.stderr))
    return obj, r.stderr


def build(verbose_regs=False, quiet=True):
    """Compile every source that changed and link libcompact_b200.so."""
    return _build(verbose_regs, quiet)


def _build(verbose_regs, quiet):
    os.makedirs(BUILD, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        results = list(ex.map(lambda s: _compile(s, verbose_regs), sources()))
    objs = [o for o, _ in results]
    if verbose_regs:
        for _, log in results:
            sys.stdout.write(log)
    if not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode:
            raise RuntimeError("link failed:\n%s%s" % (r.stdout, r.stderr))
    if not quiet:
        print("built", LIB)
    return LIB


if __name__ == "__main__":
    build(verbose_regs="-v" in sys.argv, quiet=False)
