"""openkspace_b200 -- B200-native (sm_100a) FISTA-CS reconstruction path of
OpenKSpace, behind the C-ABI of ``include/okscuda.h``.

The compute lives in ``libokscuda.so`` (hand-written CUDA in ``csrc/``); the
Python modules here are the host side: device contexts and arrays
(``device``), the drop-in strategy mirror (``strategy``) and the seeded
synthetic inputs used by tests and the benchmark (``synth``).
"""
from ._lib import OksError  # noqa: F401
from .device import Context, DeviceArray  # noqa: F401

__all__ = ["Context", "DeviceArray", "OksError"]
