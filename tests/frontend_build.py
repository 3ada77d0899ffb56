"""Builds tests/cpp/frontend_driver against the header-only C++ front end and
the CUDA library (used by test_frontend.py and test_gpu_frontend.py)."""
import subprocess
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
SRC = ROOT / "tests" / "cpp" / "frontend_driver.cpp"
OUT = ROOT / "tests" / "cpp" / "_build" / "frontend_driver"


def cuda_home() -> Path:
    from libnt_b200.build import nvcc
    return Path(nvcc()).resolve().parent.parent


def build(syntax_only: bool = False) -> Path:
    cuda = cuda_home()
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Werror", f"-I{ROOT / 'include'}",
           f"-I{ROOT / 'libnt_b200' / 'include'}", f"-I{cuda / 'include'}", str(SRC)]
    if syntax_only:
        cmd.append("-fsyntax-only")
    else:
        OUT.parent.mkdir(parents=True, exist_ok=True)
        cmd += [f"-L{ROOT / 'libnt_b200'}", "-llnt_cuda", f"-L{cuda / 'lib64'}", "-lcudart",
                "-Wl,-rpath,$ORIGIN/../../../libnt_b200", f"-Wl,-rpath,{cuda / 'lib64'}", "-o", str(OUT)]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return OUT
