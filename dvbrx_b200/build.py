"""Build ``libdvbrx_b200.so`` in-tree with nvcc for sm_100a.

    python -m dvbrx_b200.build        (or dvbrx_b200.build.build())

Every CUDA source is compiled with ``-gencode arch=compute_100a,code=sm_100a``
and linked with the static CUDA runtime into one shared library beside this
file; the ptxas resource report of the last build is kept in
``_build/ptxas.log``.  Sources compile in parallel, and an object is rebuilt
only when its source or a header it includes (nvcc's dependency file) is newer
than the object.
"""
import concurrent.futures
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libdvbrx_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xptxas", "-v",
                     "-I" + CSRC, "-I" + os.path.join(ROOT, "include")]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu"))) + sorted(glob.glob(os.path.join(CSRC, "*.cpp")))


def _deps(obj):
    """Files an object was built from (its nvcc dependency file), or None."""
    d = obj + ".d"
    if not os.path.exists(d):
        return None
    text = open(d).read().replace("\\\n", " ")
    files = []
    for line in text.splitlines():
        if ":" in line:
            files += line.split(":", 1)[1].split()
    return files


def _obj_stale(src, obj):
    if not os.path.exists(obj):
        return True
    deps = _deps(obj)
    if deps is None:
        return True
    t = os.path.getmtime(obj)
    return any(not os.path.exists(p) or os.path.getmtime(p) > t for p in deps + [src, os.path.abspath(__file__)])


def _compile(src, obj):
    cmd = [nvcc()] + NVCC_FLAGS + ["-MD", "-MF", obj + ".d", "-c", src, "-o", obj]
    if src.endswith(".cpp"):
        cmd = [nvcc(), "-x", "cu"] + NVCC_FLAGS + ["-MD", "-MF", obj + ".d", "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    return src, r.returncode, " ".join(cmd) + "\n" + r.stdout + r.stderr


def build(force=False, verbose=False):
    """Compile (in parallel, stale objects only) and link the library;
    returns its path."""
    os.makedirs(BUILD, exist_ok=True)
    srcs = sources()
    objs = [os.path.join(BUILD, os.path.basename(src) + ".o") for src in srcs]
    todo = [(s, o) for s, o in zip(srcs, objs) if force or _obj_stale(s, o)]
    if not todo and os.path.exists(LIB) and all(os.path.getmtime(o) <= os.path.getmtime(LIB) for o in objs):
        return LIB
    log = []
    jobs = max(1, min(len(todo), os.cpu_count() or 1))
    with concurrent.futures.ThreadPoolExecutor(jobs) as ex:
        for src, rc, text in ex.map(lambda so: _compile(*so), todo):
            log.append(text)
            if rc != 0:
                sys.stderr.write(text)
                raise RuntimeError("nvcc failed on " + src)
    tmp = LIB + ".tmp"
    cmd = [nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", tmp] + objs
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("link failed")
    os.replace(tmp, LIB)
    # the resource report of every object compiled this time, appended to the kept ones
    plog = os.path.join(BUILD, "ptxas.log")
    with open(plog, "a" if os.path.exists(plog) and not force else "w") as f:
        f.write("\n".join(log))
    if verbose:
        print("built", LIB, "(%d objects compiled)" % len(todo))
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
