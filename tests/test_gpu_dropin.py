"""Drop-in check: a program written against halloc.h only, compiled with
-rdc=true and device-linked with libhalloc.a, the way halloc's own samples
build (halloc samples/common.mk, README "Compiling Your Program")."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DROPIN = os.path.join(ROOT, "tests", "dropin")


def _build(name: str, lib: str, defines: list, force: bool) -> str:
    from halloc_b200.build import ARCH, INCLUDE, nvcc
    src = os.path.join(DROPIN, name + ".cu")
    exe = os.path.join(DROPIN, "_build", name)
    if not force and os.path.exists(exe) and os.path.getmtime(exe) >= max(
            os.path.getmtime(src), os.path.getmtime(lib)):
        return exe
    os.makedirs(os.path.dirname(exe), exist_ok=True)
    obj = exe + ".o"
    subprocess.run([nvcc()] + ARCH + ["-O3", "-rdc=true", "-I" + INCLUDE] + defines +
                   ["-c", src, "-o", obj], check=True)
    subprocess.run([nvcc()] + ARCH + [obj, lib, "-o", exe], check=True)
    return exe


def build_dropin_sample(force: bool = False) -> str:
    """nvcc -rdc=true user_kernel.cu + libhalloc.a -> tests/dropin/_build."""
    from halloc_b200.build import LIB_A
    return _build("user_kernel", LIB_A, [], force)


def build_new_delete_sample(force: bool = False) -> str:
    """user_new.cu with -DHALLOC_CPP + libhalloc.a -> tests/dropin/_build."""
    from halloc_b200.build import LIB_A
    return _build("user_new", LIB_A, ["-DHALLOC_CPP"], force)


@pytest.mark.gpu
def test_device_new_delete_served_by_the_allocator(torch_cuda):
    exe = build_new_delete_sample()
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("OK"), r.stdout


@pytest.mark.gpu
def test_user_program_links_and_runs(torch_cuda):
    exe = build_dropin_sample()
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("OK"), r.stdout


REF_SAMPLES = os.path.join(DROPIN, "_build", "ref")


@pytest.mark.gpu
@pytest.mark.parametrize("name,expect", [
    ("grid-points", ["allocation performance", "free performance"]),
    ("add-strings", ["GPU allocation performance", "GPU concatenation performance",
                     "GPU freeing performance"]),
    ("random-graph", ["GPU performance"]),
])
def test_reference_sample_runs_unchanged(torch_cuda, name, expect):
    """halloc's own sample program, its source untouched, compiled against
    include/halloc.h and linked with libhalloc.a (tests/dropin/Makefile): it
    runs to the end on this allocator (the samples stop with exit(-1) on any
    CUDA error) and prints its timings."""
    exe = os.path.join(REF_SAMPLES, name)
    if not os.path.exists(exe):
        pytest.skip("built where the reference tree is present: make -C tests/dropin ref-samples")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    for line in expect:
        assert line in r.stdout, r.stdout
