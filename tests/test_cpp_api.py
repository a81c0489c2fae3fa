"""Upstream's C++ API (include/libopenntc/) compiles unchanged against libontc.so."""
import subprocess

import pytest

from tests.conftest import ROOT

SRC = ROOT / "tests" / "cpp" / "upstream_api_example.cpp"


def build_example(out_dir):
    exe = out_dir / "upstream_api_example"
    lib = ROOT / "openntc_b200"
    subprocess.run(["g++", "-std=c++20", "-O1", "-I", str(ROOT / "include"), str(SRC), "-o", str(exe),
                    f"-L{lib}", "-lontc", f"-Wl,-rpath,{lib}"], check=True)
    return exe


def test_upstream_api_example_compiles_and_links(tmp_path, lib):
    exe = build_example(tmp_path)
    assert exe.exists()


@pytest.mark.gpu
def test_upstream_api_example_runs(tmp_path, materials, lib):
    exe = build_example(tmp_path)
    r = subprocess.run([str(exe), str(materials(1024, 2, 9)), str(tmp_path / "m.ntc"), "300"], capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    assert "PSNR" in r.stdout and (tmp_path / "m.ntc").stat().st_size > 10000
