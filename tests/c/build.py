"""Builds the C drop-in caller (tests/c/dropin_caller.c) with gcc, linked
against the product library libdvbrx_b200.so:

* against this project's header (include/dvbrx_b200.h), anywhere;
* against the reference's own headers (libdvbrx/include), where the
  reference tree is given (an argument, or DVBRX_REFERENCE): the binary is
  kept in tests/c/_bin/ so that it can run on machines without that tree.

    python tests/c/build.py [reference tree]
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
LIBDIR = os.path.join(ROOT, "dvbrx_b200")
BIN = os.path.join(HERE, "_bin")
SRC = os.path.join(HERE, "dropin_caller.c")


def build(out, ref_include=None):
    """Compile and link; returns the binary's path (raises on failure)."""
    os.makedirs(os.path.dirname(out), exist_ok=True)
    inc = ["-I" + ref_include] if ref_include else ["-DUSE_B200_HEADER", "-I" + os.path.join(ROOT, "include")]
    rpath = os.path.relpath(LIBDIR, os.path.dirname(out))
    cmd = ["gcc", "-O2", "-std=c11", "-Wall", "-Wextra", "-Werror"] + inc + [SRC, "-o", out, "-L" + LIBDIR,
                                                                             "-ldvbrx_b200",
                                                                             "-Wl,-rpath,$ORIGIN/" + rpath]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return out


def reference_include(tree=None):
    tree = tree or os.environ.get("DVBRX_REFERENCE")
    if tree:
        inc = os.path.join(tree, "libdvbrx", "include")
        if os.path.exists(os.path.join(inc, "dvbrx", "ldpc.h")):
            return inc
    return None


if __name__ == "__main__":
    inc = reference_include(sys.argv[1] if len(sys.argv) > 1 else None)
    print(build(os.path.join(BIN, "dropin_own_header")))
    if inc:
        print(build(os.path.join(BIN, "dropin_ref_headers"), inc))
