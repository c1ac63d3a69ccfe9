"""Drop-in check: a program written against halloc.h only, compiled with
-rdc=true and device-linked with libhalloc.a, the way halloc's own samples
build (halloc samples/common.mk, README "Compiling Your Program")."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "dropin", "user_kernel.cu")
BIN = os.path.join(ROOT, "tests", "dropin", "_build", "user_kernel")


def build_dropin_sample(force: bool = False) -> str:
    """nvcc -rdc=true user_kernel.cu + libhalloc.a -> tests/dropin/_build."""
    from halloc_b200.build import ARCH, INCLUDE, LIB_A, nvcc
    if not force and os.path.exists(BIN) and os.path.getmtime(BIN) >= max(
            os.path.getmtime(SRC), os.path.getmtime(LIB_A)):
        return BIN
    os.makedirs(os.path.dirname(BIN), exist_ok=True)
    obj = BIN + ".o"
    subprocess.run([nvcc()] + ARCH + ["-O3", "-rdc=true", "-I" + INCLUDE, "-c", SRC, "-o", obj],
                   check=True)
    subprocess.run([nvcc()] + ARCH + [obj, LIB_A, "-o", BIN], check=True)
    return BIN


@pytest.mark.gpu
def test_user_program_links_and_runs(torch_cuda):
    exe = build_dropin_sample()
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("OK"), r.stdout
