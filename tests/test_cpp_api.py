"""The C++ host API (Grammar / Graph / Matrix / MatricesEnv, cfpq-on-gpgpu_b200/cpp)
with a CPU bitset backend: loaders, driver worklist, the environment_closure
hook and print_results against the golden fixtures.  No GPU needed."""
import os
import shutil
import subprocess

import pytest

from conftest import GOLDEN, ROOT

PKG = os.path.join(ROOT, "cfpq-on-gpgpu_b200")
CASES = sorted(d for d in os.listdir(GOLDEN) if os.path.isdir(os.path.join(GOLDEN, d)))


@pytest.fixture(scope="module")
def cpu_backend(tmp_path_factory):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    lib = os.path.join(PKG, "lib", "libcfpq_b200.so")
    if not os.path.exists(lib):
        pytest.skip("library not built")
    exe = str(tmp_path_factory.mktemp("cpp") / "cpu_backend_main")
    # the graph loader is the library's (cfpq_graph_load, host code: no GPU needed)
    subprocess.run([cxx, "-O2", "-std=c++17", "-Wall", "-I", os.path.join(PKG, "cpp"),
                    "-I", os.path.join(ROOT, "include"), "-o", exe,
                    os.path.join(ROOT, "tests", "cpp", "cpu_backend_main.cpp"),
                    os.path.join(PKG, "cpp", "Grammar.cpp"), os.path.join(PKG, "cpp", "Graph.cpp"),
                    "-L", os.path.dirname(lib), "-lcfpq_b200", f"-Wl,-rpath,{os.path.dirname(lib)}"], check=True)
    return exe


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("mode", ["worklist", "hook"])
def test_cpp_driver_matches_golden(oracle, cpu_backend, case, mode, tmp_path):
    d = os.path.join(GOLDEN, case)
    out = tmp_path / "answer.txt"
    p = subprocess.run([cpu_backend, os.path.join(d, "grammar.txt"), os.path.join(d, "graph.txt"), str(out), mode],
                       capture_output=True, timeout=600)
    assert p.returncode == 0 and p.stderr == b""
    total, algo = (int(x) for x in p.stdout.split())
    assert total >= algo >= 0
    assert out.read_text() == open(os.path.join(d, "expected.txt")).read()


def test_b200_backend_compiles_against_the_c_abi(tmp_path):
    """B200Matrix.h + main_b200.cpp build against include/cfpq_b200.h and the
    library (link check only; running it needs a GPU)."""
    lib = os.path.join(PKG, "lib", "libcfpq_b200.so")
    if not os.path.exists(lib):
        pytest.skip("library not built")
    exe = str(tmp_path / "b200GPU")
    subprocess.run(["g++", "-O2", "-std=c++17", "-Wall", "-I", os.path.join(PKG, "cpp"), "-I",
                    os.path.join(ROOT, "include"), "-o", exe, os.path.join(PKG, "cpp", "main_b200.cpp"),
                    os.path.join(PKG, "cpp", "Grammar.cpp"), os.path.join(PKG, "cpp", "Graph.cpp"),
                    "-L", os.path.dirname(lib), "-lcfpq_b200", f"-Wl,-rpath,{os.path.dirname(lib)}"], check=True)
    assert os.path.exists(exe)
