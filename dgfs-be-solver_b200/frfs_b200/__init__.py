# -*- coding: utf-8 -*-
"""frfs_b200: B200-native DGFS hot path behind frfs's solver-side API.

Python host code for the fast-spectral VHS collision operator and the FR-DG
advection residual of the DGFS solver (Ehsan-Roohi/DGFS-BE-Solver, package
``frfs``).  The numerics run in ``libdgfs_b200.so`` (hand-written CUDA for
sm_100a, C ABI in include/dgfs_b200.h); this package mirrors frfs's
scattering-model, velocity-mesh, system and stepper interfaces around it.
"""

__version__ = '0.1.0'
