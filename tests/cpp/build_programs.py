"""Builds the C++ driver programs of tests/cpp against libats_b200.so (test
infrastructure). vbd_dag and async_dag also link the CPU oracle, whose per-step entry
points are their host implementation of the VBD tasks."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

SOURCES = ["heft_case.cpp", "vbd_dag.cpp", "async_dag.cpp", "launch_modes.cpp", "example2_sequence.cpp"]
WITH_ORACLE = {"vbd_dag.cpp", "async_dag.cpp"}


def _stale(out, deps):
    return not os.path.exists(out) or any(os.path.getmtime(d) > os.path.getmtime(out) for d in deps)


def build_programs():
    from libatssim_b200 import build
    from oracle import ats_oracle
    lib = build.build()
    ats_oracle.build()
    out_dir = os.path.join(build.BUILD, "tests")
    os.makedirs(out_dir, exist_ok=True)
    oracle_dir = os.path.dirname(ats_oracle.LIB_PATH)
    outs = {}
    for src in SOURCES:
        path = os.path.join(HERE, src)
        exe = os.path.join(out_dir, src[:-4])
        deps = [path, lib, os.path.join(ROOT, "include", "ats_launcher.hpp"), os.path.join(ROOT, "include", "ats_cloth.h")]
        extra = []
        if src in WITH_ORACLE:
            deps.append(ats_oracle.LIB_PATH)
            extra = ["-L" + oracle_dir, "-lats_oracle", "-Wl,-rpath," + oracle_dir]
        if _stale(exe, deps):
            cmd = ([os.environ.get("CXX", "g++"), "-O2", "-std=c++20", "-I" + os.path.join(ROOT, "include"), "-o", exe,
                    path, "-L" + build.LIBDIR, "-lats_b200", "-Wl,-rpath," + build.LIBDIR] + extra + ["-lpthread"])
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        outs[src[:-4]] = exe
    return outs


if __name__ == "__main__":
    print(build_programs())
