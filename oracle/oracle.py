"""ctypes front end for the C oracle (TEST INFRASTRUCTURE).

Loads oracle/libgpz_oracle.so (built by oracle/Makefile) and exposes numpy /
bytes helpers.  Only tests, the smoke check and the CPU-baseline leg of the
benchmark import this module; the CUDA product path never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgpz_oracle.so")
MEMBER_BYTES = 128 * 1024
# the 10-byte member header of deflate.rs:962-980 (GPZIP_HEADER, parallel_decompress.rs:29)
GZIP_HEADER = bytes([0x1F, 0x8B, 0x08, 0x00, 0x00, 0x00, 0x00, 0x00, 0x00, 0xFF])

_lib = None


def build() -> str:
    """Compile the oracle with its Makefile (gcc; no CUDA needed)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        u8p = ctypes.c_void_p
        L.gpzo_hash3.argtypes = [u8p, ctypes.c_uint32]
        L.gpzo_hash3.restype = ctypes.c_uint32
        L.gpzo_match_find.argtypes = [u8p, ctypes.c_uint32, u8p]
        L.gpzo_match_find.restype = ctypes.c_int
        L.gpzo_greedy_walk.argtypes = [u8p, u8p, ctypes.c_uint32, u8p]
        L.gpzo_greedy_walk.restype = ctypes.c_size_t
        L.gpzo_build_code_lengths.argtypes = [u8p, ctypes.c_int, ctypes.c_int, u8p]
        L.gpzo_build_code_lengths.restype = ctypes.c_int
        L.gpzo_encode_block_fast.argtypes = [u8p, ctypes.c_size_t, u8p, ctypes.c_size_t]
        L.gpzo_encode_block_fast.restype = ctypes.c_size_t
        L.gpzo_encode_block_fixed.argtypes = [u8p, ctypes.c_size_t, u8p, ctypes.c_size_t]
        L.gpzo_encode_block_fixed.restype = ctypes.c_size_t
        L.gpzo_crc32.argtypes = [u8p, ctypes.c_size_t]
        L.gpzo_crc32.restype = ctypes.c_uint32
        L.gpzo_gzip_member.argtypes = [u8p, ctypes.c_uint32, u8p, ctypes.c_size_t]
        L.gpzo_gzip_member.restype = ctypes.c_size_t
        L.gpzo_gzip_chunk.argtypes = [u8p, ctypes.c_size_t, ctypes.c_size_t, u8p, ctypes.c_size_t,
                                      ctypes.c_int]
        L.gpzo_gzip_chunk.restype = ctypes.c_size_t
        L.gpzo_member_bound.argtypes = [ctypes.c_size_t]
        L.gpzo_member_bound.restype = ctypes.c_size_t
        L.gpzo_brute_lz77.argtypes = [u8p, ctypes.c_uint32, ctypes.c_uint32, u8p]
        L.gpzo_brute_lz77.restype = None
        L.gpzcpu_gzip_chunks.argtypes = [u8p, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_int,
                                         ctypes.c_int, u8p, ctypes.c_size_t]
        L.gpzcpu_gzip_chunks.restype = ctypes.c_size_t
        L.gpzo_zstd_chunk.argtypes = [u8p, ctypes.c_size_t, ctypes.c_size_t, u8p, ctypes.c_size_t]
        L.gpzo_zstd_chunk.restype = ctypes.c_size_t
        L.gpzo_zstd_bound.argtypes = [ctypes.c_size_t, ctypes.c_size_t]
        L.gpzo_zstd_bound.restype = ctypes.c_size_t
        _lib = L
    return _lib


def _u8(data) -> np.ndarray:
    if isinstance(data, np.ndarray):
        return np.ascontiguousarray(data, dtype=np.uint8)
    return np.frombuffer(bytes(data), dtype=np.uint8)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p) if a.size else ctypes.c_void_p(0)


def match_find(data) -> np.ndarray:
    """Per-position packed tokens (u32 per input byte)."""
    a = _u8(data)
    pp = np.zeros(max(a.size, 1), dtype=np.uint32)
    if a.size and lib().gpzo_match_find(_ptr(a), a.size, _ptr(pp)) != 0:
        raise MemoryError("oracle match_find allocation failed")
    return pp[:a.size]


def brute_lz77(data, window: int = 4096) -> np.ndarray:
    a = _u8(data)
    pp = np.zeros(max(a.size, 1), dtype=np.uint32)
    if a.size:
        lib().gpzo_brute_lz77(_ptr(a), a.size, window, _ptr(pp))
    return pp[:a.size]


def greedy_walk(pp: np.ndarray, data) -> np.ndarray:
    a = _u8(data)
    pp = np.ascontiguousarray(pp, dtype=np.uint32)
    out = np.zeros(max(a.size, 1), dtype=np.uint32)
    k = lib().gpzo_greedy_walk(_ptr(pp), _ptr(a), a.size, _ptr(out)) if a.size else 0
    return out[:k]


def tokens(data) -> np.ndarray:
    """Walked token stream for one member."""
    return greedy_walk(match_find(data), data)


def build_code_lengths(freq, max_bits: int):
    f = np.ascontiguousarray(freq, dtype=np.uint32)
    lens = np.zeros(f.size, dtype=np.uint8)
    ok = lib().gpzo_build_code_lengths(_ptr(f), f.size, max_bits, _ptr(lens))
    return lens if ok else None


def encode_block_fast(toks: np.ndarray) -> bytes:
    t = np.ascontiguousarray(toks, dtype=np.uint32)
    cap = 1100 + 2 * t.size * 6 + 64
    out = np.zeros(cap, dtype=np.uint8)
    k = lib().gpzo_encode_block_fast(_ptr(t), t.size, _ptr(out), cap)
    if k == 0:
        raise RuntimeError("oracle encode overflow")
    return out[:k].tobytes()


def encode_block_fixed(toks: np.ndarray) -> bytes:
    """write_fixed_block_fast alone (deflate.rs:763-799)."""
    t = np.ascontiguousarray(toks, dtype=np.uint32)
    cap = 64 + 4 * t.size + 64
    out = np.zeros(cap, dtype=np.uint8)
    k = lib().gpzo_encode_block_fixed(_ptr(t), t.size, _ptr(out), cap)
    if k == 0:
        raise RuntimeError("oracle encode overflow")
    return out[:k].tobytes()


def gzip_member_fixed(data) -> bytes:
    """A gzip member whose DEFLATE block is the fixed-Huffman one
    (deflate.rs:962-980 around write_fixed_block_fast)."""
    import struct
    a = _u8(data)
    body = encode_block_fixed(tokens(a)) if a.size else encode_block_fixed(np.zeros(0, np.uint32))
    return GZIP_HEADER + body + struct.pack("<II", crc32(a), a.size & 0xFFFFFFFF)


def gzip_chunk_fixed(data, member_bytes: int = MEMBER_BYTES) -> bytes:
    a = _u8(data)
    if a.size <= member_bytes:
        return gzip_member_fixed(a)
    return b"".join(gzip_member_fixed(a[o:o + member_bytes]) for o in range(0, a.size, member_bytes))


def crc32(data) -> int:
    a = _u8(data)
    return lib().gpzo_crc32(_ptr(a), a.size)


def gzip_member(data) -> bytes:
    a = _u8(data)
    cap = lib().gpzo_member_bound(a.size)
    out = np.zeros(cap, dtype=np.uint8)
    k = lib().gpzo_gzip_member(_ptr(a), a.size, _ptr(out), cap)
    if k == 0:
        raise RuntimeError("oracle gzip_member failed")
    return out[:k].tobytes()


def gzip_chunk(data, member_bytes: int = MEMBER_BYTES, threads: int = 1) -> bytes:
    """gzip_chunk_fn: concatenated members of member_bytes each."""
    a = _u8(data)
    nmem = max(1, -(-a.size // member_bytes))
    cap = nmem * lib().gpzo_member_bound(member_bytes)
    out = np.zeros(cap, dtype=np.uint8)
    k = lib().gpzo_gzip_chunk(_ptr(a), a.size, member_bytes, _ptr(out), cap, threads)
    if k == 0:
        raise RuntimeError("oracle gzip_chunk failed")
    return out[:k].tobytes()


def cpu_gzip_chunks(data, chunk: int = 2 << 20, level: int = 5, threads: int = 1) -> bytes:
    """gpzip-cpu-equivalent: zlib 1.3 gzip member per chunk, all threads."""
    a = _u8(data)
    nch = max(1, -(-a.size // chunk))
    cap = a.size + a.size // 100 + 1024 * nch + 4096
    out = np.zeros(cap, dtype=np.uint8)
    k = lib().gpzcpu_gzip_chunks(_ptr(a), a.size, chunk, level, threads, _ptr(out), cap)
    if k == 0:
        raise RuntimeError("cpu gzip failed")
    return out[:k].tobytes()


def zstd_chunk(data, member_bytes: int = MEMBER_BYTES) -> bytes:
    """The GPU zstd codec's frame for one chunk (oracle/zstd_frame.c)."""
    a = _u8(data)
    cap = lib().gpzo_zstd_bound(a.size, member_bytes)
    out = np.zeros(cap, dtype=np.uint8)
    k = lib().gpzo_zstd_chunk(_ptr(a), a.size, member_bytes, _ptr(out), cap)
    if k == 0:
        raise RuntimeError("oracle zstd_chunk failed")
    return out[:k].tobytes()


_zstd = None


def zstd_lib():
    """libzstd (the system's shared library, no header needed): the
    independent decoder the zstd frames are checked with, and the CPU
    baseline's encoder."""
    global _zstd
    if _zstd is None:
        z = ctypes.CDLL("libzstd.so.1")
        z.ZSTD_decompress.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t]
        z.ZSTD_decompress.restype = ctypes.c_size_t
        z.ZSTD_compress.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
        z.ZSTD_compress.restype = ctypes.c_size_t
        z.ZSTD_compressBound.argtypes = [ctypes.c_size_t]
        z.ZSTD_compressBound.restype = ctypes.c_size_t
        z.ZSTD_isError.argtypes = [ctypes.c_size_t]
        z.ZSTD_isError.restype = ctypes.c_uint
        z.ZSTD_getErrorName.argtypes = [ctypes.c_size_t]
        z.ZSTD_getErrorName.restype = ctypes.c_char_p
        _zstd = z
    return _zstd


def zstd_decompress(frames: bytes, size: int) -> bytes:
    """libzstd's decoder over one or more concatenated frames of `size`
    decompressed bytes in total; raises on any decoding error."""
    z = zstd_lib()
    src = np.frombuffer(frames, dtype=np.uint8)
    dst = np.zeros(max(size, 1), dtype=np.uint8)
    r = z.ZSTD_decompress(_ptr(dst), dst.size, _ptr(src), src.size)
    if z.ZSTD_isError(r):
        raise ValueError("libzstd: " + z.ZSTD_getErrorName(r).decode())
    if r != size:
        raise ValueError(f"libzstd decoded {r} bytes, expected {size}")
    return dst[:size].tobytes()


def zstd_compress(data, level: int = 3) -> bytes:
    """libzstd's own encoder (one frame), the gpzip-cpu zstd path's engine."""
    z = zstd_lib()
    a = _u8(data)
    cap = z.ZSTD_compressBound(a.size)
    out = np.zeros(max(cap, 1), dtype=np.uint8)
    r = z.ZSTD_compress(_ptr(out), cap, _ptr(a), a.size, level)
    if z.ZSTD_isError(r):
        raise ValueError("libzstd: " + z.ZSTD_getErrorName(r).decode())
    return out[:r].tobytes()
