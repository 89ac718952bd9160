# -*- coding: utf-8 -*-
"""Properties of the FR-DG oracle on CPU (free-stream preservation and
conservation), the checks frfs's discretisation guarantees."""

import numpy as np

from helpers import config, dg_setup
from frfs_b200 import mesh as mgen


def _periodic_cfg():
    cfg = config('relax0d-n16')
    cfg.set('solver', 'order', 2)
    return cfg


def test_free_stream_preservation():
    cfg = _periodic_cfg()
    m = mgen.quad_box(3, 3, 0.0, 1.0, 0.0, 1.0, periodic_x=True,
                      periodic_y=True, jitter=0.2, seed=4)
    dg, sh, geo, vm = dg_setup(cfg, m)
    f = np.exp(-np.sum(vm.cv()**2, axis=0))
    u = np.broadcast_to(f[None, :, None], (sh.nupts, vm.vsize(),
                                           geo.neles)).copy()
    R = dg.rhs(u)
    assert np.max(np.abs(R)) < 1e-11*np.max(np.abs(f))*vm.L()


def test_periodic_residual_conserves_mass():
    cfg = _periodic_cfg()
    m = mgen.quad_box(3, 2, 0.0, 1.0, 0.0, 0.5, periodic_x=True,
                      periodic_y=True, jitter=0.15, seed=2)
    dg, sh, geo, vm = dg_setup(cfg, m)
    rng = np.random.default_rng(0)
    u = rng.uniform(0.5, 1.5, (sh.nupts, vm.vsize(), geo.neles))
    R = dg.rhs(u)
    # quadrature of the residual over the domain: sum w |J| R = 0
    from frfs_b200.quadratures import gauss_legendre
    z, w = gauss_legendre(3)
    w2 = np.array([w[i]*w[j] for j in range(3) for i in range(3)])
    djac = geo.djac_at(sh.upts)
    tot = np.einsum('u,ue,uve->v', w2, djac, R)
    scale = np.einsum('u,ue,uve->v', w2, djac, np.abs(R))
    assert np.all(np.abs(tot) < 1e-11*scale.max())
