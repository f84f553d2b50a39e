"""B200-native implementation of OpenSWPC's viscoelastic FDM time step.

The compute path is the CUDA library ``lib/libswpc_gpu.so`` (C ABI in
``include/swpc_gpu.h``); this package is its host-side driver.
"""
__version__ = "0.1.0"
