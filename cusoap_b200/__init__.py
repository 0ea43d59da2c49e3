"""B200-native SOAP descriptor generator (drop-in for ``cusoap.SOAP``).

``from cusoap_b200 import SOAP`` -- the compute path is the CUDA library
``libsoapb200.so`` (sm_100a), reached through its C ABI (include/soapb200.h).
"""
from .soap import SOAP
from .xyz import read_xyz

__all__ = ["SOAP", "read_xyz"]
__version__ = "0.1.0"
