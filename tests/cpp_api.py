"""Builds tests/cpp/grid_api.cpp (a driver of the C++ mirror of the
reference API, include/deepgreen.hpp) against libdeepgreen.so."""
import subprocess
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
LIB_DIR = ROOT / "deep-green_b200" / "lib"


def build(outdir: Path) -> Path:
    exe = Path(outdir) / "grid_api"
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", str(ROOT / "include"),
           str(ROOT / "tests" / "cpp" / "grid_api.cpp"), "-o", str(exe), "-L", str(LIB_DIR), "-ldeepgreen",
           f"-Wl,-rpath,{LIB_DIR}", "-Wl,--allow-shlib-undefined"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode:
        raise RuntimeError(r.stderr[-4000:])
    return exe
