# -*- coding: utf-8 -*-
"""FR operators and element geometry against the reference's own output
(fixtures from frfs/shapes.py and frfs/solvers/base/elements.py)."""

import numpy as np
import pytest

from conftest import GOLDEN
from frfs_b200 import mesh as mgen
from frfs_b200.elements import ElementGeometry
from frfs_b200.shapes import QuadShape


@pytest.mark.parametrize('order', [1, 2, 3])
def test_quad_operators_match_reference(order):
    g = np.load(f'{GOLDEN}/ref_shape_quad_p{order}.npz')
    sh = QuadShape(order)
    np.testing.assert_allclose(sh.upts, g['upts'], atol=1e-15)
    np.testing.assert_allclose(sh.fpts, g['fpts'], atol=1e-15)
    np.testing.assert_array_equal(sh.norm_fpts, g['norm_fpts'])
    for key, expr in [('M0', 'M0'), ('M1', 'M1'), ('M2', 'M2'), ('M3', 'M3'),
                      ('M132', 'M1 - M3*M2'), ('M12', 'M12')]:
        np.testing.assert_allclose(sh.opmat(expr), g[key], rtol=0,
                                   atol=2e-14, err_msg=key)


@pytest.mark.parametrize('order,jitter', [(2, 0.2), (1, 0.15), (3, 0.1)])
def test_element_geometry_matches_reference(order, jitter):
    g = np.load(f'{GOLDEN}/ref_dg_quad_p{order}.npz')
    m = mgen.quad_box(4, 3, 0.0, 1.0, 0.0, 0.75, periodic_x=True,
                      jitter=jitter, seed=order)
    np.testing.assert_array_equal(m['spt_quad_p0'], g['spt'])
    np.testing.assert_array_equal(m['con_p0'], g['con'])
    sh = QuadShape(order)
    geo = ElementGeometry(sh, m['spt_quad_p0'])
    tol = dict(rtol=1e-13, atol=1e-14)
    np.testing.assert_allclose(geo.smat_at(sh.upts), g['smats_upts'], **tol)
    np.testing.assert_allclose(geo.rcpdjac_at(sh.upts), g['rcpdjac_upts'],
                               **tol)
    np.testing.assert_allclose(geo.ploc_upts, g['ploc_upts'], **tol)
    np.testing.assert_allclose(geo.plocfpts, g['plocfpts'], **tol)
    np.testing.assert_allclose(geo.norm_pnorm_fpts, g['norm_pnorm_fpts'],
                               **tol)
    np.testing.assert_allclose(geo.mag_pnorm_fpts, g['mag_pnorm_fpts'],
                               **tol)
    np.testing.assert_array_equal(np.array(geo.srtd_face_fpts),
                                  g['srtd_face_fpts'])
