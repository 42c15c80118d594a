"""The boundary from compiled C and C++, as an HLR-side caller would use it.

* tests/c/two_streams.c links libhlrc.so like any C program, builds and
  uploads a matrix through the C ABI and runs products of one handle on two
  CUDA streams with two workspaces (hlrc_mvm_ws), checked against the
  oracle's hlr::seq::mul_vec restatement (linked as the checker).
* The HLR-side adapter printed in INTEGRATION.md (section 2) is extracted
  and compiled against a small stand-in for the HLR / HLIBpro types
  (tests/c/mock_hlr.hh), then run on a two-level block matrix.
Without a GPU the programs are compiled, linked and run in their dry mode."""
import re
import subprocess

import pytest

from conftest import ROOT

CUDA = "/usr/local/cuda"
LIBS = [f"-L{ROOT / 'hlr_b200'}", "-lhlrc", f"-L{ROOT / 'oracle'}", "-loracle", f"-L{CUDA}/lib64", "-lcudart", "-lm",
        f"-Wl,-rpath,{ROOT / 'hlr_b200'}:{ROOT / 'oracle'}:{CUDA}/lib64"]


def _oracle_built():
    import oracle
    oracle.build()


def _compile(cc, src, exe, extra=()):
    _oracle_built()
    cmd = [cc, "-O2", "-Wall", f"-I{ROOT / 'include'}", f"-I{CUDA}/include", *extra, str(src), "-o", str(exe), *LIBS]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def _run(exe, *args, timeout=600):
    r = subprocess.run([str(exe), *args], capture_output=True, text=True, timeout=timeout)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout


def test_c_caller_compiles_links_and_plans(tmp_path):
    exe = tmp_path / "two_streams"
    _compile("gcc", ROOT / "tests" / "c" / "two_streams.c", exe, ["-std=c11"])
    out = _run(exe, "--dry")
    assert "dry run ok" in out


@pytest.mark.gpu
def test_c_caller_two_streams_two_workspaces(tmp_path):
    exe = tmp_path / "two_streams"
    _compile("gcc", ROOT / "tests" / "c" / "two_streams.c", exe, ["-std=c11"])
    out = _run(exe)
    worst = float(re.search(r"worst (\S+)", out).group(1))
    assert worst <= 1e-13, out


def _adapter_source(tmp_path):
    """The first C++ block of INTEGRATION.md section 2, with the HLR includes
    replaced by the stand-in header."""
    text = (ROOT / "INTEGRATION.md").read_text()
    sec = text[text.index("## 2."):]
    code = re.search(r"```cpp\n(.*?)```", sec, re.S).group(1)
    code = re.sub(r"#include <hlr/[^>]*>\n", "", code)
    code = code.replace("#include <hlrc.h>", '#include "hlrc.h"\n#include "mock_hlr.hh"')
    hdr = tmp_path / "arith.hh"
    hdr.write_text(code)
    return hdr


def _build_adapter(tmp_path):
    _adapter_source(tmp_path)
    exe = tmp_path / "adapter"
    _compile("g++", ROOT / "tests" / "c" / "adapter_main.cpp", exe,
             ["-std=c++17", f"-I{tmp_path}", f"-I{ROOT / 'tests' / 'c'}"])
    return exe


def test_integration_adapter_compiles(tmp_path):
    exe = _build_adapter(tmp_path)
    assert "flattened 4 leaves" in _run(exe, "--dry")


@pytest.mark.gpu
def test_integration_adapter_runs(tmp_path):
    exe = _build_adapter(tmp_path)
    out = _run(exe)
    err = float(re.search(r"rel\. error (\S+)", out).group(1))
    assert err <= 1e-13, out
