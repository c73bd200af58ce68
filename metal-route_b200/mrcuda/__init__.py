"""mrcuda — B200-native batched shortest-path engine for metalroute.

The compute lives in libmr_cuda.so (hand-written sm_100a CUDA kernels and a
C++ runtime behind include/mr_cuda.h); this package is its Python binding and
the plain data types of the reference's contract.
"""
from .types import (  # noqa: F401
    BOARD_EDGE_NEG_X,
    BOARD_EDGE_NEG_Y,
    BOARD_EDGE_POS_X,
    BOARD_EDGE_POS_Y,
    BOARD_TRACE_NODE,
    BOARD_VIA_NODE,
    COST_MAX,
    OBSTACLE,
    Dims,
    Grid,
    IsolatedRouteRequest,
    IsolatedRouteWindow,
    connection_group_ids,
    group_of,
    NetEndpoints,
)
from .api import (  # noqa: F401
    BackendUnavailable,
    Batch,
    Board,
    BoardRoute,
    Busy,
    CudaIsolatedProvider,
    Engine,
    InvalidArgument,
    InvalidEndpoint,
    IsolatedBatchResult,
    IterationLimit,
    LimitExceeded,
    MalformedGrid,
    Negotiation,
    Server,
    OutOfMemory,
    RouterError,
    exported_symbols,
    load_library,
    net_windows,
)
