"""halloc's own correctness suite on this allocator.

The programs of halloc's tst/corr (checkptr, freeslabs, prob-checkptr, test)
are compiled from the reference tree unchanged against include/halloc.h and
libhalloc.a (tests/dropin/Makefile, target ref-tests) and run here with the
arguments of halloc's suite driver, tst/corr/run-all-tests.pl:20-69.  A
program passes when it exits 0: each calls exit(-1) when a pointer is NULL,
when two blocks overlap or a block is shorter than asked (its harness sorts
all live pointers and checks the gaps, tst/common/common.cu:465-529), and on
any CUDA error.

One change of size: run-all-tests.pl gives prob-checkptr 16,384 tries
(divided by the iterations per try); here it gets 128, so the suite takes
about two minutes instead of an hour.
"""
import math
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "tests", "dropin", "_build", "ref")
MEMORY = 512 * 1024 * 1024  # run-all-tests.pl:10

pytestmark = pytest.mark.gpu


def _run(name: str, *args: str, timeout: int = 300) -> subprocess.CompletedProcess:
    exe = os.path.join(BIN, name)
    if not os.path.exists(exe):
        pytest.skip("built where the reference tree is present: make -C tests/dropin ref-tests")
    return subprocess.run([exe, *args], capture_output=True, text=True, timeout=timeout)


def checkptr_cases() -> list:
    """The size sweep of run-all-tests.pl:20-44: 16 B to 32 KiB, a quarter of
    the memory in blocks of each size up to 2 KiB, an eighth above (sizes above
    3 KiB go to CUDA's allocator, as in halloc)."""
    cases, size, step = [], 16, 8
    while size <= 32 * 1024:
        fraction = 0.25 if size <= 2 * 1024 else 0.125
        n = math.floor(fraction * MEMORY / size)
        if n:
            cases.append((size, n))
        if size >= 16 * 1024:
            step = 16 * 1024
        elif size >= 2 * 1024:
            step = 2 * 1024
        elif size >= 256:
            step = 256
        elif size >= 64:
            step = 16
        else:
            step = 8
        size += step
    return cases


@pytest.mark.parametrize("size,n", checkptr_cases(), ids=lambda v: str(v))
def test_checkptr(torch_cuda, size, n):
    r = _run("checkptr", "-l1", "-t4", f"-s{size}", f"-n{n}", "-D0", f"-m{MEMORY}")
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]


def test_freeslabs(torch_cuda):
    """Every size from 16 B to 1 KiB in turn fills 40 % of the memory and frees
    it again: slabs must come back free to serve the next size."""
    r = _run("freeslabs", f"-m{MEMORY}", "-D0")
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]


PROB_SIZES = [  # run-all-tests.pl:59-67
    ("-l4", "-n1048576", "-s8", "-S64", "-duniform"),
    ("-l1", "-n1048576", "-s8", "-S256", "-duniform"),
    ("-l4", "-n1048576", "-s8", "-S256", "-dexpequal"),
    ("-l1", "-n65536", "-s8", "-S3072", "-duniform"),
    ("-l4", "-n131072", "-s8", "-S3072", "-dexpequal"),
]


@pytest.mark.parametrize("group", [0, 5, 10])
@pytest.mark.parametrize("niters", [1, 5])
@pytest.mark.parametrize("sizes", PROB_SIZES, ids=lambda s: "".join(s[:1] + s[3:]))
def test_prob_checkptr(torch_cuda, group, niters, sizes):
    """Threads allocate and free at random over many launches (f = F = 0.5,
    e = 0.75); after every launch all live blocks are checked."""
    ntries = math.ceil(128 / niters)
    r = _run("prob-checkptr", f"-i{niters}", f"-t{ntries}", "-f0.5", "-F0.5", "-e0.75",
             f"-g{group}", *sizes, "-D0", f"-m{MEMORY}")
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]


def test_corr_test_program(torch_cuda):
    """tst/corr/test: 2 M blocks of 16 B allocated, sorted and checked for
    16 bytes of room each (and written), then the timing tests."""
    r = _run("test")
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "test PASSED" in r.stdout and "FAILED" not in r.stdout, r.stdout


def test_phase_extfrag_program(torch_cuda):
    """tst/perf/phase-extfrag: halloc's harness calls ha_extfrag(false) and
    ha_extfrag(true) after every launch of the phase workload; both are
    fractions of the free slab memory."""
    r = _run("phase-extfrag", "-f0.95", "-F0.05", "-e0.91", f"-m{MEMORY}", "-g5", "-n1048576",
             "-l1", "-s8", "-S256", "-i1", "-t8", "-D0")
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    rows = [line.split() for line in r.stdout.splitlines()
            if line.startswith("external fragmentation")]
    assert len(rows) == 8, r.stdout
    for row in rows:
        real, ideal = float(row[3]), float(row[4])
        assert 0.0 <= real <= 1.0 and 0.0 <= ideal <= 1.0, row


@pytest.mark.parametrize("prog,line", [("throughput", "pair throughput"),
                                       ("latency", "malloc latency")])
def test_perf_program_runs(torch_cuda, prog, line):
    """tst/perf/throughput (all mallocs of a launch, then all frees) and
    tst/perf/latency (clock around each call) with their default options:
    1 M threads, 4 blocks of 16 B each, 8 tries.  Each checks every pointer
    for NULL after its malloc launch and stops on one."""
    r = _run(prog, "-D0", f"-m{MEMORY}")
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert line in r.stdout, r.stdout
