"""B200-native query path for hnswlib indexes.

``Index`` / ``BFIndex`` mirror ``hnswlib.Index`` / ``hnswlib.BFIndex`` for
loading saved indexes and answering ``knn_query`` on the GPU; the kernels live
in libhnswgpu.so (C ABI: include/hnswgpu.h).
"""
from .index import BFIndex, Index  # noqa: F401

__version__ = "0.1.0"
