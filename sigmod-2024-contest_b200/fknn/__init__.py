"""fknn -- B200 filtered k-nearest-neighbour engine (host side).

The compute path is libfknn.so (hand-written sm_100a CUDA kernels behind the
C ABI of include/fknn.h); this package is its Python binding and a mirror of
the reference's entry points (see api.py).
"""
from ._lib import (FKNN_ECUDA, FKNN_EINVAL, FKNN_ENODEV, FKNN_ENOMEM, FKNN_ETIMEOUT, FKNN_EUNSUPPORTED, FKNN_OK,
                   MODE_BF16_RERANK, MODE_EXACT_FP32, MODE_FP8_RERANK, FknnError, LIB_PATH, load)
from .api import (DIM, K, Bruteforce, GraphSearcher, Index, Router, Server, SQ8SymmetricQuantizer, bruteforce,
                  bruteforce_subgraph, read_base_file, read_groundtruth, read_query_file, save_knn,
                  sorted_query_order)

__all__ = [
    "Index", "GraphSearcher", "Router", "Server", "Bruteforce", "bruteforce", "bruteforce_subgraph", "SQ8SymmetricQuantizer",
    "read_base_file", "read_query_file", "sorted_query_order", "save_knn", "read_groundtruth", "FknnError", "load",
    "LIB_PATH", "DIM", "K", "MODE_EXACT_FP32", "MODE_BF16_RERANK", "MODE_FP8_RERANK", "FKNN_OK", "FKNN_EINVAL",
    "FKNN_ENOMEM", "FKNN_ECUDA", "FKNN_ETIMEOUT", "FKNN_EUNSUPPORTED", "FKNN_ENODEV",
]
