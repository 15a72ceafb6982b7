"""The header-only C++ facade (include/inq_b200.hpp): compiles against the C ABI here, and on a GPU
reproduces the reference's ks_hamiltonian known answers (ks_hamiltonian.hpp:297-445)."""

import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "inq_b200")


def _compile(out):
    src = os.path.join(ROOT, "tests", "cpp", "ks_hamiltonian_kat.cpp")
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    cmd = ["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), "-I", os.path.join(cuda, "include"), src,
           "-o", out, "-L", LIBDIR, "-linqb200", f"-Wl,-rpath,{LIBDIR}", "-L", os.path.join(cuda, "lib64"), "-lcudart",
           f"-Wl,-rpath,{os.path.join(cuda, 'lib64')}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


def test_facade_compiles(tmp_path):
    from inq_b200 import _lib
    _lib.load()  # the library exists
    _compile(str(tmp_path / "kat"))


@pytest.mark.gpu
def test_facade_known_answers(tmp_path):
    exe = _compile(str(tmp_path / "kat"))
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "harmonic oscillator: 0.00514" in r.stdout
    assert "wrapped device buffers: 0 values differ" in r.stdout
