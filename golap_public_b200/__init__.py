"""B200-native GOLAP query hot path: compressed column chunks decoded in shared
memory and fused with min/max pruning, filtering, hash-join probing and
hash aggregation (libgx.so, sm_100a)."""
from ._lib import GxError, lib  # noqa: F401

__all__ = ["GxError", "lib"]
