"""Build libpsgpu.so (sm_100a) in-tree.

    python -m polyspectrum_b200.build [--force] [--ptxas-verbose] [--kbench]

Each translation unit compiles in its own nvcc process (the FFT kernels are
heavily unrolled); objects go to polyspectrum_b200/_build/, the shared library
to polyspectrum_b200/libpsgpu.so.  The library links the CUDA runtime
statically and depends on no torch symbol.  The command-line driver
(driver/ps_run.c, plain C over the C-ABI) is linked against it as
polyspectrum_b200/ps_run, and the ini-file generator (driver/ps_create_ini.c) as
polyspectrum_b200/ps_create_ini.  --kbench also builds polyspectrum_b200/ps_kbench, a
stand-alone timing harness of the hot passes (csrc/ps_kbench.cu).
"""
from __future__ import annotations

import argparse
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OUT_DIR = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libpsgpu.so")
DRIVER_SRC = os.path.join(PKG, "driver", "ps_run.c")
DRIVER = os.path.join(PKG, "ps_run")
KBENCH = os.path.join(PKG, "ps_kbench")
CREATE_INI_SRC = os.path.join(PKG, "driver", "ps_create_ini.c")
CREATE_INI = os.path.join(PKG, "ps_create_ini")
SOURCES = ["ps_api.cu", "ps_inst_f32.cu", "ps_inst_f64.cu", "ps_inst_f32_mixed.cu", "ps_inst_f64_mixed.cu",
           "ps_noalloc.cu"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _deps() -> list[str]:
    return (glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cuh"))
            + glob.glob(os.path.join(ROOT, "include", "*.h")))


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(p) <= t for p in _deps())


def build_driver(force: bool = False) -> str:
    """gcc the C driver against libpsgpu.so (rpath $ORIGIN: the two stay side by side)."""
    if (not force and os.path.exists(DRIVER)
            and os.path.getmtime(DRIVER) >= max(os.path.getmtime(DRIVER_SRC), os.path.getmtime(LIB),
                                                os.path.getmtime(os.path.join(ROOT, "include", "ps_gpu.h")))):
        return DRIVER
    tmp = DRIVER + ".tmp"
    subprocess.run(["gcc", "-std=c99", "-O2", "-Wall", "-Wextra", "-o", tmp, DRIVER_SRC, "-L", PKG, "-lpsgpu",
                    "-Wl,-rpath,$ORIGIN", "-lm"], check=True)
    os.replace(tmp, DRIVER)
    build_create_ini()
    return DRIVER


def build_create_ini() -> str:
    """gcc the ini-file generator (plain C, no library)."""
    if os.path.exists(CREATE_INI) and os.path.getmtime(CREATE_INI) >= os.path.getmtime(CREATE_INI_SRC):
        return CREATE_INI
    tmp = CREATE_INI + ".tmp"
    subprocess.run(["gcc", "-std=c99", "-O2", "-Wall", "-Wextra", "-o", tmp, CREATE_INI_SRC], check=True)
    os.replace(tmp, CREATE_INI)
    return CREATE_INI


def build(force: bool = False, ptxas_verbose: bool = False, quiet: bool = False) -> str:
    if not force and up_to_date():
        build_driver()
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    exe = nvcc()
    procs = []
    objs = []
    for src in SOURCES:
        obj = os.path.join(OUT_DIR, src.replace(".cu", ".o"))
        objs.append(obj)
        cmd = [exe, *FLAGS, "-c", os.path.join(CSRC, src), "-o", obj]
        if ptxas_verbose:
            cmd += ["-Xptxas", "-v"]
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                                            text=True)))
    failed = False
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            failed = True
            sys.stderr.write(f"nvcc failed for {src}:\n{out}\n")
        elif out and (ptxas_verbose or not quiet):
            lines = [ln for ln in out.splitlines() if "Wno-deprecated" not in ln]
            if lines:
                sys.stdout.write("\n".join(lines) + "\n")
    if failed:
        raise RuntimeError("libpsgpu build failed")
    tmp = LIB + ".tmp"
    subprocess.run([exe, *ARCH, "-shared", "-cudart", "static", *objs, "-o", tmp], check=True)
    os.replace(tmp, LIB)
    build_driver(force=True)
    return LIB


def build_kbench() -> str:
    """nvcc the stand-alone kernel timing harness (no library link)."""
    tmp = KBENCH + ".tmp"
    subprocess.run([nvcc(), *FLAGS, "-o", tmp, os.path.join(CSRC, "ps_kbench.cu")], check=True)
    os.replace(tmp, KBENCH)
    return KBENCH


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas-verbose", action="store_true")
    ap.add_argument("--kbench", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, ptxas_verbose=a.ptxas_verbose))
    if a.kbench:
        print(build_kbench())


if __name__ == "__main__":
    main()
