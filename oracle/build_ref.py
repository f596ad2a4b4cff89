"""Build recipe for ``oracle/_ref/libbbhx_ref.so`` (test infrastructure only).

Compiles the reference's own CPU implementation of the waveform -> likelihood path
directly from its sources under the reference checkout (``src/bbhx/cutils``), each
``.cu`` file as C++ the way the reference CPU backend does
(``src/bbhx/cutils/CMakeLists.txt:388-396``), together with

* ``oracle/shims/lapacke.h``   -- DGTSV stand-in (no LAPACK in this image),
* ``oracle/shims/Detector.hpp`` -- lisatools orbit-table stand-in,
* ``oracle/ref_capi.cpp``       -- extern "C" forwarding layer for ctypes.

Nothing is copied out of the reference tree; outputs go only to ``oracle/_ref/``.
The library is single-threaded, as the reference CPU build is (its OpenMP pragmas are
inert without ``-fopenmp``).  ``-march=x86-64-v3`` keeps the binary runnable on any
AVX2 host.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")
OUT = os.path.join(OUT_DIR, "libbbhx_ref.so")
# Location of the reference checkout this recipe compiles from: BBHX_REFERENCE_ROOT, else the
# checkout directory of the build container.  The golden-fixture scripts and
# oracle/make_qnm_table.py read it from here; nothing outside oracle/ and tests/golden/ does.
REF_ROOT = os.environ.get("BBHX_REFERENCE_ROOT", "/root/reference")
CUTILS = os.path.join(REF_ROOT, "src", "bbhx", "cutils")
SOURCES = [
    "PhenomHMWaveform.cu",
    "Response.cu",
    "Interpolate.cu",
    "WaveformBuild.cu",
    "Likelihood.cu",
]
FLAGS = ["-O3", "-march=x86-64-v3", "-std=c++17", "-fPIC", "-w"]


def reference_available() -> bool:
    return all(os.path.isfile(os.path.join(CUTILS, s)) for s in SOURCES)


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile the reference CPU path; returns the library path."""
    if not reference_available():
        raise FileNotFoundError(f"reference sources not found under {CUTILS}")
    os.makedirs(OUT_DIR, exist_ok=True)
    deps = [os.path.join(CUTILS, s) for s in SOURCES] + [
        os.path.join(HERE, "ref_capi.cpp"),
        os.path.join(HERE, "shims", "lapacke.h"),
        os.path.join(HERE, "shims", "Detector.hpp"),
        os.path.abspath(__file__),
    ]
    if (not force) and os.path.isfile(OUT):
        t_out = os.path.getmtime(OUT)
        if all(os.path.getmtime(d) <= t_out for d in deps):
            return OUT
    objs = []
    for src in SOURCES + ["ref_capi.cpp"]:
        path = os.path.join(CUTILS, src) if src.endswith(".cu") else os.path.join(HERE, src)
        obj = os.path.join(OUT_DIR, os.path.splitext(src)[0] + ".o")
        cmd = ["g++", *FLAGS, "-I", os.path.join(HERE, "shims"), "-I", CUTILS, "-x", "c++",
               "-c", path, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        objs.append(obj)
    cmd = ["g++", "-shared", "-o", OUT, *objs]
    subprocess.run(cmd, check=True)
    for o in objs:
        os.remove(o)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
