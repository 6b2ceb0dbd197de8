"""B200-native epsilon-grid distance self-join (drop-in for algorithm 3 of
mgowanlock/gpu_self_join).

The compute path is the in-tree native library ``libgpuselfjoin.so``
(hand-written sm_100a CUDA behind the C ABI of include/gpuselfjoin.h); this
package only binds it.
"""

from .gdsjoingpu import gdsjoin  # noqa: F401
from .selfjoin import JoinConfig, SelfJoin, threshold  # noqa: F401
