"""Compiles tests/cpp/parity.cpp against the C++ host layer and libraspagpu.so (shared by the CPU and GPU tests)."""

import os
import shutil
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "parity.cpp")
OUT = os.path.join(ROOT, "tests", "cpp", "_build", "parity")


def compile_parity() -> str:
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else shutil.which("g++")
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    lib_dir = os.path.join(ROOT, "raspa3_b200")
    cmd = [cxx, "-std=c++20", "-O2", "-Wall", "-o", OUT, SRC, f"-I{os.path.join(ROOT, 'include')}",
           f"-L{lib_dir}", "-lraspagpu", f"-Wl,-rpath,{lib_dir}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(r.stdout + r.stderr)
    return OUT
