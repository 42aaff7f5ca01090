#!/usr/bin/env python3
"""Builds the CLAST reference itself for the host CPU -- test infrastructure only.

Recipe: every translation unit of the reference (the flat source directory:
--ref, or CLAST_REFERENCE_DIR, or the build container's mount point) is compiled with g++ against Thrust's sequential CPP
device system, so thrust::device_vector storage is host memory and every
Thrust algorithm runs on the CPU.  The reference sources are read where they
lie and are not edited on disk; the only rewrite is mechanical and happens on
the text fed to the compiler:

  * `kernel<<<grid, block>>>(args)` becomes `clast_cpu_launch(grid, block, kernel, args)`
    (oracle/refshim/cuda_cpu_shim.h runs the kernel body over the grid);
  * templated comparators that Thrust now calls with two different tuple types
    get a second template parameter (same body);
  * the read2bit functor (SRead2bit.cuh:8,19) returns its (key, flag) pair by
    value: as shipped it returns thrust::tie() of its own locals, references
    that dangle once it returns.  The GPU build tolerated that undefined
    behaviour; a host compiler does not.  The arithmetic is unchanged.

Boost is not installed; oracle/refshim/boost/lexical_cast.hpp stands in for
the one Boost function the reference calls.  oracle/refshim/shim_alloc.cpp
pads every Thrust allocation with 'N' bytes so the reference's few
out-of-bounds reads see a defined base.  Output goes only to
oracle/_ref/ (git-ignored): the rewritten text under _ref/src/ and the binary
_ref/clast_ref, a drop-in of the reference's `clast` command line.

Usage: python oracle/build_ref.py [--ref DIR] [--jobs N]
"""
import argparse
import concurrent.futures as cf
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_REF = "/root/reference"  # where the build container mounts the reference sources
OUT = os.path.join(HERE, "_ref")
SRC = os.path.join(OUT, "src")
SHIM = os.path.join(HERE, "refshim")
CUDA_INC = "/usr/local/cuda/include"

# CTest.cu is the MODE_TEST debug dumper (off in the shipped build).
SKIP = {"CTest.cu"}

LAUNCH = re.compile(r"(\w+)\s*<<<\s*(.*?)\s*>>>\s*\(", re.S)
# `template <class Tuple> ... operator() (const Tuple& tuple1, const Tuple& tuple2)`
CMP = re.compile(
    r"template\s*<\s*class\s+Tuple\s*>(\s*__device__\s+bool\s+operator\(\)\s*\(\s*)"
    r"const\s+Tuple\s*&\s*tuple1\s*,\s*const\s+Tuple\s*&\s*tuple2\s*\)", re.S)


READ2BIT_SIG = "__device__ Tuple operator() (const char chr, Tuple tuple)"
READ2BIT_RET = "return thrust::tie(input, flg);"


def rewrite(text):
    if "struct read2bit" in text:
        assert READ2BIT_SIG in text and READ2BIT_RET in text, "read2bit changed upstream"
        text = text.replace(READ2BIT_SIG,
                            "__device__ thrust::tuple<long, char> operator() (const char chr, Tuple tuple)")
        text = text.replace(READ2BIT_RET, "return thrust::make_tuple(input, flg);")
    text = LAUNCH.sub(lambda m: "clast_cpu_launch(%s, %s, " % (m.group(2), m.group(1)), text)
    text = CMP.sub(lambda m: "template <class Tuple, class Tuple2>%sconst Tuple& tuple1, const Tuple2& tuple2)"
                   % m.group(1), text)
    return text


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("CLAST_REFERENCE_DIR", DEFAULT_REF),
                    help="the reference's source directory (also CLAST_REFERENCE_DIR)")
    ap.add_argument("--jobs", type=int, default=os.cpu_count() or 4)
    ap.add_argument("--cxx", default="g++")
    args = ap.parse_args()
    ref = os.path.abspath(args.ref)
    if not os.path.isdir(ref):
        print("reference sources not found at %s; nothing built" % ref)
        return 0
    os.makedirs(SRC, exist_ok=True)
    units = []
    for name in sorted(os.listdir(ref)):
        path = os.path.join(ref, name)
        if name in SKIP or not os.path.isfile(path):
            continue
        if name.endswith((".cuh", ".hpp")):
            text = open(path, encoding="latin-1").read()
            new = rewrite(text)
            if new != text:  # only headers that needed the rewrite are shadowed
                open(os.path.join(SRC, name), "w", encoding="latin-1").write(new)
        elif name.endswith((".cu", ".cpp")):
            text = open(path, encoding="latin-1").read()
            out = os.path.join(SRC, os.path.splitext(name)[0] + ".cpp")
            open(out, "w", encoding="latin-1").write(rewrite(text))
            units.append(out)
    flags = ["-std=c++17", "-O2", "-fopenmp", "-w",
             "-DTHRUST_DEVICE_SYSTEM=THRUST_DEVICE_SYSTEM_CPP",
             "-DTHRUST_HOST_SYSTEM=THRUST_HOST_SYSTEM_CPP",
             "-I", SHIM, "-I", CUDA_INC, "-iquote", SRC, "-iquote", ref,
             "-include", os.path.join(SHIM, "cuda_cpu_shim.h")]

    def compile_one(src):
        obj = os.path.join(SRC, os.path.basename(src)[:-4] + ".o")
        r = subprocess.run([args.cxx] + flags + ["-c", src, "-o", obj],
                           capture_output=True, text=True)
        return src, obj, r

    units.append(os.path.join(SHIM, "shim_alloc.cpp"))
    objs, failed = [], []
    with cf.ThreadPoolExecutor(args.jobs) as ex:
        for src, obj, r in ex.map(compile_one, units):
            if r.returncode != 0:
                failed.append((src, r.stderr))
            else:
                objs.append(obj)
    for src, err in failed:
        print("FAILED %s\n%s" % (src, err[-4000:]), file=sys.stderr)
    if failed:
        return 1
    exe = os.path.join(OUT, "clast_ref")
    r = subprocess.run([args.cxx, "-fopenmp", "-o", exe] + objs, capture_output=True, text=True)
    if r.returncode != 0:
        print(r.stderr[-4000:], file=sys.stderr)
        return 1
    print("built %s from %d translation units" % (exe, len(objs)))
    return 0


if __name__ == "__main__":
    sys.exit(main())
