"""evoc on B200: the kNN-graph hot path of evoc-rs as CUDA for sm_100a.

Host-side mirror of the evoc-rs kNN interface over the C ABI in
include/evoc_gpu.h (libevoc_gpu.so, built in-tree).
"""
from ._lib import build, context, header_symbols  # noqa: F401
from .backend import ComputeBackend, CudaBackend, make_backend  # noqa: F401
from .boruvka import parallel_boruvka  # noqa: F401
from .graph import neighbor_graph_csr, neighbor_graph_matrix, smooth_knn_dist  # noqa: F401
from .label_prop import label_prop_loop, label_propagation_init, node_embedding  # noqa: F401
from .knn import (  # noqa: F401
    BackendError,
    EmbeddingData,
    EmptyData,
    InvalidNeighbors,
    KnnError,
    KnnGraphOptions,
    autotune,
    knn_graph,
    knn_graph_batch,
    knn_graph_batch_device,
    knn_graph_device,
    knn_graph_ref,
    transform_distances_float,
)
