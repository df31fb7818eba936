"""Build ``libhippymfem_b200.so`` in-tree with nvcc for sm_100a.

    python hippymfem_b200/build.py            # build if a source is newer than the .so
    python hippymfem_b200/build.py --force    # rebuild
    python hippymfem_b200/build.py --ptxas    # also print registers / spills / smem

(Run as a script: importing the package would load the library being rebuilt.)

Objects go to ``hippymfem_b200/_build`` (git-ignored); the library lands next to this
file so that it travels with the source tree.
"""

import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
OUT = os.path.join(HERE, "libhippymfem_b200.so")
BUILD = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-I" + INCLUDE]
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-pthread", "-I" + INCLUDE]


def nvcc():
    cand = os.environ.get("NVCC") or os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"),
                                                  "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def sources():
    cu = sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))
    cpp = sorted(f for f in os.listdir(CSRC) if f.endswith(".cpp"))
    return cu, cpp


def _stale():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE)]
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("command failed: %s" % " ".join(cmd[:3]))
    return r.stdout + r.stderr


def build(force=False, verbose=False, ptxas=False):
    """Compile every source and link the shared library; returns its path."""
    if not force and not ptxas and not _stale():
        return OUT
    os.makedirs(BUILD, exist_ok=True)
    cu, cpp = sources()
    objs = []
    report = []
    for f in cu:
        o = os.path.join(BUILD, f + ".o")
        extra = ["-Xptxas", "-v"] if ptxas else []
        report.append(_run([nvcc()] + NVCC_FLAGS + ARCH + extra + ["-c", os.path.join(CSRC, f),
                                                                  "-o", o], verbose))
        objs.append(o)
    for f in cpp:
        o = os.path.join(BUILD, f + ".o")
        _run(["g++"] + CXX_FLAGS + ["-c", os.path.join(CSRC, f), "-o", o], verbose)
        objs.append(o)
    tmp = OUT + ".tmp"
    _run([nvcc(), "-shared"] + ARCH + ["-o", tmp] + objs + ["-lcudart", "-lpthread"], verbose)
    os.replace(tmp, OUT)
    if ptxas:
        print("\n".join(report))
    return OUT


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose, ptxas=a.ptxas))
