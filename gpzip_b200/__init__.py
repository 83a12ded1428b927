"""B200-native (sm_100a) gzip compression path for gpzip.

The compute path is libgpz.so (CUDA kernels + C ABI, include/gpz.h);
``native`` binds it with ctypes and ``codec`` mirrors the reference's
chunk-codec interface on top of it.
"""
