"""cggraph_b200 -- a B200 (sm_100a) graph engine behind CGgraph's interface.

BFS, SSSP, CC and PageRank over a binary CSR run in hand-written CUDA kernels
(libcgb200.so, C ABI in include/cgb200.h); this package is the host-side
mirror of the reference's SINGLE_GPU interface (GraphDeviceWorklist,
main_partition, load_binFile, checkBinResult).
"""
from ._lib import CgbError, LIB_PATH, VALUE_MAX  # noqa: F401
from .engine import (  # noqa: F401
    Algorithm_type,
    Batch,
    CSR_Result_type,
    DEFAULT_TUNING,
    Engine_type,
    Graph,
    GraphB200,
    OrderMethod,
    Server,
    VertexValue_MAX,
    checkBinResult,
    chunglu_draws_for_edges,
    chunglu_expected_edges,
    chunglu_weight_offset,
    load_binFile,
    main_partition,
    make_options,
    memory_info,
    memory_reserve,
    memory_trim,
    reorder_graph,
    save_binArray,
    trimmed_mean_ms,
)
