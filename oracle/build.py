"""ORACLE / TEST INFRASTRUCTURE ONLY: builds the CPU checkers.

  oracle/libscoracle.so  -- the plain-C restatement (sc_oracle.c)
  oracle/_ref/libscref.so -- the reference's own hot-path sources compiled
                             where they lie (only when the reference tree is
                             present; on machines without it the prebuilt
                             library, if any, is used as is)
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
# Where the reference's source tree is read from (its src/ and include/);
# SIMCORE_REFERENCE_TREE overrides the default location.
REFERENCE_TREE = os.environ.get("SIMCORE_REFERENCE_TREE", "/root/reference")


def _cc():
    # The system compiler (the image's CC wrapper lacks the OpenMP spec file).
    for c in ("/usr/bin/gcc", "gcc"):
        if shutil.which(c):
            return c
    raise RuntimeError("no C compiler found")


def build_oracle(verbose=False):
    out = os.path.join(HERE, "libscoracle.so")
    srcs = [os.path.join(HERE, f) for f in ("sc_oracle.c", "sc_oracle_insert.c")]
    hdrs = [os.path.join(HERE, h) for h in ("sc_oracle.h", "sc_philox.h")]
    if os.path.exists(out) and all(os.path.getmtime(out) >= os.path.getmtime(p)
                                   for p in srcs + hdrs):
        return out
    cmd = [_cc(), "-O2", "-std=c99", "-fPIC", "-shared", "-ffp-contract=off",
           "-o", out] + srcs + ["-lm"]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    return out


def build_reference(verbose=False, jobs=8):
    """Builds oracle/_ref/libscref.so from the reference tree if present."""
    if not os.path.isdir(os.path.join(REFERENCE_TREE, "src")):
        return None
    cmd = ["make", "-s", "-C", os.path.join(HERE, "ref"), "-j%d" % jobs,
           "REF=" + REFERENCE_TREE, "OUT=" + os.path.join(HERE, "_ref"),
           "REFCXX=" + ("/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++")]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    return os.path.join(HERE, "_ref", "libscref.so")


if __name__ == "__main__":
    print(build_oracle(verbose=True))
    print(build_reference(verbose=True))
    sys.exit(0)
