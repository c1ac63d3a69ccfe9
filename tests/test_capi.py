"""The C ABI library and the drop-in static library: they load, export every
symbol the headers declare, and keep the reference's layouts.  CPU only (no
call that needs a GPU)."""
import ctypes
import os
import re
import subprocess

import pytest

import halloc_b200 as H

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions(header: str) -> list:
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int|double|uint32_t|void)\s+\**(ha_\w+)\s*\(",
                                 text, flags=re.M)))


def test_header_declares_abi():
    names = declared_functions("halloc_c.h")
    assert "ha_init_c" in names and "ha_trace_c" in names and len(names) >= 16


def test_shared_library_exports_every_declared_symbol():
    lib = H.load()
    missing = [n for n in declared_functions("halloc_c.h") if not hasattr(lib, n)]
    assert missing == []


def test_static_library_keeps_reference_symbols():
    """A halloc program links against libhalloc.a unchanged: the device and
    host entry points carry the reference's C++ mangled names."""
    a = os.path.join(ROOT, "halloc_b200", "libhalloc.a")
    out = subprocess.run(["nm", a], capture_output=True, text=True, check=True).stdout
    for sym in ("_Z8hamallocm", "_Z6hafreePv", "_Z7ha_init13halloc_opts_t",
                "_Z11ha_shutdownv", "_Z10ha_extfragb"):
        assert re.search(rf"\bT {sym}\b", out), sym


def test_options_layout_matches_halloc_opts_t():
    """x86-64 layout of halloc_opts_t: size_t + 4 doubles + int, 48 bytes."""
    assert ctypes.sizeof(H._COpts) == 48
    assert H._COpts.sb_sz_sh.offset == 40
    d = H.HallocOpts()
    assert (d.memory, d.halloc_fraction, d.busy_fraction, d.roomy_fraction,
            d.sparse_fraction, d.sb_sz_sh) == (512 << 20, 0.75, 0.835, 0.6, 0.012, 22)


def test_stats_layout():
    assert ctypes.sizeof(H._CStats) == 5 * 8 + 8 * 4 + 32 * 4 + 2 * 4 + 8 + 16 * 4 + 2 * 4


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setattr(H, "SO_PATH", str(tmp_path / "absent.so"))
    monkeypatch.setattr(H, "_lib", None)
    with pytest.raises(H.HallocError):
        H.load()


def test_pyfast_binding_checks_arguments():
    """The CPython binding of the host-buffer loop is built beside the
    library and reaches the same C ABI function as ctypes: the same argument
    errors, before any CUDA call."""
    import halloc_b200 as H
    assert H._pyfast is not None
    with pytest.raises(TypeError):
        H._pyfast.throughput_host(0, 0, 16)
    with pytest.raises(OverflowError):
        H._pyfast.throughput_host(0, 0, 1 << 32, 1, 128, 1, 1, 0, 0, 0, 0)
    with pytest.raises(OverflowError):
        H._pyfast.throughput_host(-1, 0, 16, 1, 128, 1, 1, 0, 0, 0, 0)
    # d_out NULL: HA_EINVAL from both bindings
    args = (0, 0, 16, 1, 128, 1, 1, 0, 8, 0, 0)
    assert H._pyfast.throughput_host(*args) == H.load().ha_throughput_host_ex_c(*args) == -1


def test_probe_counters_only_in_instrumented_builds():
    """The probe counters (ha_probe_stats_c) are compiled in only with
    -DHA_PROBE_STATS: the normal library does not export them, and the
    probe-counter tool stops before any GPU work, naming the build flag."""
    from halloc_b200 import probestats
    assert not hasattr(H.load(), "ha_probe_stats_c")
    with pytest.raises(SystemExit) as e:
        probestats.run(1, True)
    assert "HA_PROBE_STATS" in str(e.value)
