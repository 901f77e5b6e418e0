"""Build the CUDA library libqcbc_gpu.so in-tree for sm_100a.

Steps:
1. Generate csrc/_gen/qnm_table.h: the IMRPhenomD quasi-normal-mode table
   (final spin, fring, fdamp; IMRPhenomD_internals.h:176-640 of the QuickCBC
   reference) read from the reference tree given by QCBC_REFERENCE (default: a
   `reference` directory beside this repository).  The generated file is a
   build output and is not committed.
   When the reference tree is absent the existing generated file is reused.
2. nvcc -gencode arch=compute_100a,code=sm_100a for the kernels and the C ABI.

Usage:  python -m quickcbc_b200.build [--force]
"""
from __future__ import annotations

import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
GEN = os.path.join(CSRC, "_gen")
LIB = os.path.join(HERE, "libqcbc_gpu.so")
SOURCES = ["qcbc_kernels.cu", "qcbc_capi.cu", "qcbc_serve.cu", "qcbc_hetspace.cu", "qcbc_ptstep.cu", "qcbc_ingest.cu"]
HEADERS = ["qcbc_device.cuh", "qcbc_kernels.cuh", "qcbc_hetspace.h", "qcbc_ptstep.h", "qcbc_ingest_dev.h"]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall", "--expt-relaxed-constexpr"]


def reference_dir() -> str:
    return os.environ.get("QCBC_REFERENCE") or os.path.normpath(os.path.join(HERE, "..", "..", "reference"))


def gen_qnm(force: bool = False) -> str:
    out = os.path.join(GEN, "qnm_table.h")
    src = os.path.join(reference_dir(), "IMRPhenomD_internals.h")
    if os.path.exists(out) and not force:
        return out
    if not os.path.exists(src):
        if os.path.exists(out):
            return out
        raise FileNotFoundError(
            f"{src} not found: the QNM table is read from the QuickCBC reference at build time "
            "(set QCBC_REFERENCE to the reference checkout)")
    text = open(src).read()
    arrays = {}
    for name in ("QNMData_a", "QNMData_fring", "QNMData_fdamp"):
        m = re.search(r"static const double " + name + r"\[\]\s*=\s*\{(.*?)\};", text, re.S)
        if not m:
            raise RuntimeError(f"{name} not found in {src}")
        body = m.group(1).replace("\\", " ")
        arrays[name] = [float(x) for x in re.findall(r"[-+]?[0-9]*\.?[0-9]+(?:[eE][-+]?[0-9]+)?", body)]
    n = len(arrays["QNMData_a"])
    if any(len(v) != n for v in arrays.values()):
        raise RuntimeError("QNM tables differ in length")
    os.makedirs(GEN, exist_ok=True)
    with open(out, "w") as f:
        f.write("// generated by quickcbc_b200/build.py from the reference's IMRPhenomD_internals.h\n")
        f.write("#pragma once\n")
        f.write(f"#define QCBC_QNM_N {n}\n")
        for cname, key in (("QCBC_QNM_A", "QNMData_a"), ("QCBC_QNM_FRING", "QNMData_fring"),
                           ("QCBC_QNM_FDAMP", "QNMData_fdamp")):
            f.write(f"static const double {cname}[{n}] = {{{','.join(repr(v) for v in arrays[key])}}};\n")
    return out


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.exists(d) and os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    qnm = gen_qnm()
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS] + [qnm, __file__]
    deps += [os.path.join(HERE, "..", "include", h) for h in ("qcbc_gpu.h", "qcbc_quickcbc.h", "qcbc_serve.h",
                                                                   "qcbc_ingest.h")]
    if not force and not _stale(LIB, deps):
        return LIB
    nvcc = os.environ.get("NVCC", "nvcc")
    objs = []
    for s in SOURCES:
        obj = os.path.join(GEN, s.replace(".cu", ".o"))
        cmd = [nvcc, *NVCC_FLAGS, "-c", os.path.join(CSRC, s), "-o", obj]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        objs.append(obj)
    cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-Xlinker", "-Bsymbolic", "-o", LIB, *objs]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
