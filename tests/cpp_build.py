"""Helper for the tests: compile tests/cpp/drop_in.cpp against the
reference-path headers in include/imresh and libimresh_b200.so (and the CUDA
runtime, for the program's own device buffers)."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def build_drop_in(out_dir: str) -> str:
    exe = os.path.join(out_dir, "drop_in")
    lib_dir = os.path.join(ROOT, "imresh_b200", "lib")
    cmd = ["g++", "-std=c++14", "-O1", "-I", os.path.join(ROOT, "include", "imresh"),
           "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include",
           os.path.join(ROOT, "tests", "cpp", "drop_in.cpp"), "-L", lib_dir, "-limresh_b200",
           "-Wl,-rpath," + lib_dir, "-L", "/usr/local/cuda/lib64", "-lcudart",
           "-Wl,-rpath,/usr/local/cuda/lib64", "-lpthread", "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe
