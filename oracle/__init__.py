# -*- coding: utf-8 -*-
"""CPU oracle for the DGFS hot path -- TEST INFRASTRUCTURE ONLY.

This package restates, in FP64 numpy, the reference's algorithm for the
fast-spectral VHS collision operator and the FR-DG advection residual
(Ehsan-Roohi/DGFS-BE-Solver, package ``frfs``).  Every function cites the
reference ``file:line`` it follows.

It is a checker, never a product path: only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may
import it.  The B200 package fails loudly when its CUDA library is missing
and never falls back to this code.

Pinning
-------
Inputs are pinned to fixtures produced by the reference's own numpy code
(``tests/golden/make_golden.py``: velocity mesh, radial and spherical
quadrature, VHS prefactor, Maxwellian initial states, quadrilateral operator
matrices).  The collision operator itself runs on PyCUDA + cuFFT in the
reference and cannot execute here, so ``Q(f)`` is pinned by
(a) an independent direct-sum evaluation of the same discrete formula
(``vhs.vhs_direct``), (b) the invariants of the operator (mass, momentum and
energy conservation to spectral accuracy, Q(Maxwellian) ~ 0) and (c) the
BKW exact solution for Maxwell molecules.  The FFT boundary itself (cuFFT in
the reference) has no golden vectors in the reference, so bit-level parity at
that boundary is unpinned.
"""
