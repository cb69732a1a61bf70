"""The C++ host layer (raspa3_b200/host/raspa_b200.hpp): compiles and links here; its parity program runs on a GPU."""

import subprocess

import pytest

from cpp_build import compile_parity


def test_host_layer_compiles_and_links():
    assert compile_parity()


@pytest.mark.gpu
def test_cpp_parity_program_on_gpu():
    exe = compile_parity()
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "PASSED" in r.stdout
