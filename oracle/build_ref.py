"""Build the reference's own CPU scan (src/torch/torch_scan_cpu.h) into oracle/_ref/.

The reference path compiles from a single header that needs only torch and
OpenMP, so it is built here from the sources where they lie in the reference
checkout (never copied).  Output goes to oracle/_ref/ only.  Usage:

    python oracle/build_ref.py [--ref /path/to/reference]

The checkout is found from --ref, else the TCUSCAN_REFERENCE environment
variable, else a directory named ``reference`` next to this repository.

The built module is test infrastructure: tests/golden/make_golden.py uses it to
pin the oracle, and bench.py's CPU baseline times it.  Machines without the
reference checkout only load the prebuilt .so.
"""
import argparse
import glob
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")


def reference_root(ref=None):
    """The reference checkout: `ref`, else $TCUSCAN_REFERENCE, else the
    ``reference`` directory beside this repository; None if none exists."""
    for cand in (ref, os.environ.get("TCUSCAN_REFERENCE"),
                 os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")):
        if cand and os.path.isdir(os.path.join(cand, "src")):
            return cand
    return None


def built_module_path():
    hits = sorted(glob.glob(os.path.join(OUT, "tcuscan_ref_cpu*.so")))
    return hits[0] if hits else None


def build(ref_root=None, verbose=False):
    ref_root = reference_root(ref_root)
    if ref_root is None:
        raise FileNotFoundError("reference checkout not found (pass --ref or set TCUSCAN_REFERENCE)")
    header_dir = os.path.join(ref_root, "src", "torch")
    if not os.path.exists(os.path.join(header_dir, "torch_scan_cpu.h")):
        raise FileNotFoundError(f"reference CPU scan header not found under {header_dir}")
    os.makedirs(OUT, exist_ok=True)
    # /opt/gcc's g++ lacks libgomp.spec; the system g++ links OpenMP.
    if os.path.exists("/usr/bin/g++"):
        os.environ["CXX"] = "/usr/bin/g++"
        os.environ["CC"] = "/usr/bin/gcc"
    from torch.utils.cpp_extension import load

    load(
        name="tcuscan_ref_cpu",
        sources=[os.path.join(HERE, "ref_scan_cpu_binding.cpp")],
        extra_include_paths=[header_dir],
        extra_cflags=["-O3", "-fopenmp"],
        extra_ldflags=["-fopenmp"],
        build_directory=OUT,
        verbose=verbose,
    )
    return built_module_path()


def load_module():
    """Import the prebuilt reference module from oracle/_ref (no rebuild)."""
    path = built_module_path()
    if path is None:
        raise ImportError("oracle/_ref/tcuscan_ref_cpu*.so is not built; run oracle/build_ref.py")
    import importlib.util

    import torch  # noqa: F401  (libc10 must be loaded first)

    spec = importlib.util.spec_from_file_location("tcuscan_ref_cpu", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=None)
    ap.add_argument("-v", action="store_true")
    a = ap.parse_args()
    p = build(a.ref, a.v)
    print(p)
    sys.exit(0 if p else 1)
