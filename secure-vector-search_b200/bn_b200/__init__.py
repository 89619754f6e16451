"""B200 (sm_100a) backend of the Braverman-Newman scoring path.

`capi` binds the C ABI of include/bn_b200.h; the library is built in-tree by
secure-vector-search_b200/build.py.
"""
from . import capi  # noqa: F401
