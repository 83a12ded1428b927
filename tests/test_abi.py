"""The C ABI library without a GPU: it loads, exports every symbol that
include/gpz.h declares, and its argument checks and pure host functions
answer without touching a device (no compute calls here)."""
import ctypes
import os
import re
import shutil
import subprocess

import pytest

from gpzip_b200 import build, native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "gpz.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    return sorted(set(re.findall(r"GPZ_API\s+[\w\s\*]*?\b(gpz_\w+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    build.build()  # no-op when the in-tree library is up to date
    return native.load()


def test_header_and_binding_list_agree():
    names = declared_functions()
    assert len(names) >= 20
    assert names == sorted(native.EXPORTS)


def test_library_exports_every_declared_symbol(lib):
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_only_gpz_symbols_are_visible(lib):
    # built with hidden visibility: the dynamic symbol table holds the ABI only
    r = subprocess.run(["nm", "-D", "--defined-only", native.LIB_PATH], capture_output=True, text=True)
    if r.returncode != 0:
        pytest.skip("nm not available")
    syms = [ln.split()[-1] for ln in r.stdout.splitlines() if " T " in ln]
    assert sorted(s for s in syms if s.startswith("gpz_")) == declared_functions()


def test_strerror(lib):
    for code, name in native.STATUS.items():
        s = lib.gpz_strerror(code)
        assert s and s != b"unknown status", name
    assert lib.gpz_strerror(12345) == b"unknown status"


def test_bound_covers_worst_case(lib):
    # per member: 10 + 8 framing bytes, a dynamic header, at most 16 bits
    # per input byte (a 3-byte match costs at most 15 + 5 + 15 + 13 bits), EOB
    assert lib.gpz_bound(0) >= 18 + 8
    for n in (1, 100, 131071, 131072, 131073, 2 << 20, (2 << 20) + 1536):
        members = max(1, -(-n // 131072))
        assert lib.gpz_bound(n) >= 18 * members + 2 * n
        assert lib.gpz_bound(n) <= lib.gpz_bound(n + 131072)
    assert lib.gpz_bound_ctx(None, 5000) == lib.gpz_bound(5000)


def test_config_default(lib):
    cfg = native.Config()
    cfg.device = 7
    lib.gpz_config_default(ctypes.byref(cfg))
    assert cfg.device == 0 and cfg.member_bytes == 131072


def test_argument_checks_without_a_device(lib):
    vp = ctypes.c_void_p
    n = ctypes.c_size_t()
    assert lib.gpz_create(None, None) == 5
    cfg = native.Config()
    lib.gpz_config_default(ctypes.byref(cfg))
    h = vp()
    cfg.member_bytes = 1000  # not a multiple of 4096
    assert lib.gpz_create(ctypes.byref(cfg), ctypes.byref(h)) == 5
    cfg.member_bytes = 4 << 20  # above the 2 MiB member limit
    assert lib.gpz_create(ctypes.byref(cfg), ctypes.byref(h)) == 5
    assert lib.gpz_compress_chunk(None, None, 0, 5, None, 0, ctypes.byref(n)) == 5
    assert lib.gpz_compress_batch(None, None, 0, None) == 5
    assert lib.gpz_compress_batch_plain(None, None, 0, None) == 5
    assert lib.gpz_submit(None, None, None) == 5
    assert lib.gpz_poll(None, 0, None, 0) == 5
    assert lib.gpz_frame_host(None, None, 0) == 5
    assert lib.gpz_last_launches(None) == 0
    assert lib.gpz_last_error(None) == b"no context"
    lib.gpz_destroy(None)
    assert lib.gpz_inflate(None, None, 0, None, 0, ctypes.byref(n)) == 5
    assert lib.gpz_inflate_size(None, 10, None, ctypes.byref(n)) == 5
    assert lib.gpz_inflate_size(None, 0, None, None) == 5
    assert lib.gpz_inflate_device_ms(None) == 0.0
    # the allocation-free entry point checks its arguments before any CUDA call
    assert lib.gpz_compress_member_static(vp(16), 131073, vp(16), 1 << 20, ctypes.byref(n), None) == 5
    assert lib.gpz_compress_member_static(None, 10, vp(16), 1 << 20, ctypes.byref(n), None) == 5


def test_create_fails_loudly_without_a_gpu(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    cfg = native.Config()
    lib.gpz_config_default(ctypes.byref(cfg))
    h = ctypes.c_void_p()
    assert lib.gpz_create(ctypes.byref(cfg), ctypes.byref(h)) == 4  # GPZ_E_CUDA
    assert not h.value
    with pytest.raises(native.GpzError):
        native.Context()


def test_c_program_compiles_against_the_header(tmp_path):
    # a plain C caller builds against include/gpz.h and links libgpz.so
    cc = shutil.which("gcc") or shutil.which("cc")
    if not cc:
        pytest.skip("no C compiler")
    exe = tmp_path / "abi_roundtrip"
    r = subprocess.run([cc, "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                        os.path.join(ROOT, "tests", "c", "abi_roundtrip.c"), "-o", str(exe),
                        "-L", os.path.dirname(native.LIB_PATH), "-lgpz", "-lz",
                        "-Wl,-rpath," + os.path.dirname(native.LIB_PATH)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


@pytest.mark.gpu
def test_c_program_round_trip(tmp_path):
    # the same program run on the GPU: chunk and batch calls inflate back
    cc = shutil.which("gcc") or shutil.which("cc")
    if not cc:
        pytest.skip("no C compiler")
    build.build()
    exe = tmp_path / "abi_roundtrip"
    subprocess.run([cc, "-O1", "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "c", "abi_roundtrip.c"),
                    "-o", str(exe), "-L", os.path.dirname(native.LIB_PATH), "-lgpz", "-lz",
                    "-Wl,-rpath," + os.path.dirname(native.LIB_PATH)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
