"""B200-native radix bias-factorization walk engine (Bingo's hot path).

Per-vertex bit-group store, integer alias tables over group masses,
Philox-keyed DeepWalk / node2vec / PPR / one-hop sampling walks and batched
edge insert / delete, as hand-written sm_100a CUDA behind the C ABI in
include/bingo.h. This package is the host-side mirror of the reference's
operator interface (`Graph.build / insert / deleteE / walk`).
"""
from ._lib import BingoError, LIB_PATH, lib  # noqa: F401
from .engine import (APPS, BATCHED, DEEPWALK, NODE2VEC, PLAIN, PPR, RUN_GRAPH, SAMPLING,  # noqa: F401
                     WALK_PPR_TAIL, Graph, WalkJob, fixed16)
from . import gen  # noqa: F401
