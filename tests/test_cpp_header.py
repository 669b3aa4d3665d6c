"""The C++ drop-in header (include/calaman_b200.hpp) compiles with g++ for a
reference-style call site and links against the library; the host-only
contracts run on the CPU."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_cpp_header_compiles_links_and_runs(tmp_path):
    from calaman_g_b200 import capi

    exe = tmp_path / "header_check"
    libdir = os.path.dirname(capi.LIB_PATH)
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror",
                    "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "header_check.cpp"), "-o", str(exe),
                    "-L", libdir, "-lcalaman_b200", f"-Wl,-rpath,{libdir}"], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "header_check ok" in out.stdout
