"""barytreek_b200 — B200-native barycentric Lagrange dual-tree treecode.

The compute path is hand-written CUDA for sm_100a in ``libbarytreek_b200.so``
(sources in ``csrc/``, C ABI in ``include/barytreek_b200.h``); this package is
the Python host layer over that ABI.
"""
from ._lib import BtkError, load  # noqa: F401
from .treecode import (KIND_FIELD, KIND_POT, KIND_VEL, PREC_FP64, PREC_MIXED, HostTree, Treecode,  # noqa: F401
                       dual_tree_traversal, make_run_config, ncomp, read_run_config, split_interactions,
                       tree_construction)

__version__ = "0.1.0"
