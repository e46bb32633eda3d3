"""B200-native JPEG 2000 Part-1 decode path (host mirror of the reference's decoder API).

The directory name carries a hyphen, so entry points load it by path as the module
``jpeg2000_decoder_b200`` (see ``load`` in __graft_entry__.py, bench.py and tests/conftest.py).
Native pieces: libj2k_b200.so (host Tier-2 + sm_100a kernels + C ABI) and libj2kenc.so
(test codestream writer), built in-tree by build.py.
"""
from . import native  # noqa: F401
from .native import GpuContext, Plan, encode  # noqa: F401
