# -*- coding: utf-8 -*-
"""Host-side mirror of frfs's interfaces (CPU only, no CUDA calls)."""

import numpy as np
import pytest

from helpers import config, golden
from frfs_b200.backend import B200Backend
from frfs_b200.inifile import Inifile
from frfs_b200.quadratures import gauss_legendre_lobatto, zwgj
from frfs_b200.scattering import (DGFSScatteringModel,
                                  DGFSVHSGLLScatteringModel, subclass_where)
from frfs_b200.velocitymesh import DGFSVelocityMesh


@pytest.mark.parametrize('name', ['relax0d-n16', 'couette-n24',
                                  'channel-n32'])
def test_velocity_mesh_matches_reference(name):
    g = golden(name)
    cfg = config(name)
    vm = DGFSVelocityMesh(None, cfg)
    assert vm.L() == g['L'] and vm.cw() == g['cw']
    np.testing.assert_allclose(vm.qz(), g['qz'], rtol=0, atol=1e-14)
    np.testing.assert_allclose(vm.qw(), g['qw'], rtol=0, atol=1e-14)
    np.testing.assert_array_equal(vm.sz(), g['sz'])
    np.testing.assert_array_equal(vm.c0(), g['c0'])
    assert vm.sw() == g['sw'] and vm.u0() == g['u0'] and vm.n0() == g['n0']
    if 'cv' in g:
        np.testing.assert_array_equal(vm.cv(), g['cv'])


@pytest.mark.parametrize('name', ['relax0d-n16', 'couette-n24'])
def test_vhs_prefactor_matches_reference(name):
    g = golden(name)
    cfg = config(name)
    sm = object.__new__(DGFSVHSGLLScatteringModel)
    sm.cfg, sm.vm = cfg, DGFSVelocityMesh(None, cfg)
    sm.load_parameters()
    assert sm.prefactor == g['prefactor']
    assert sm._gamma == g['gamma']


def test_scattering_model_registry():
    assert subclass_where(DGFSScatteringModel, scattering_model='vhs-gll') \
        is DGFSVHSGLLScatteringModel


def test_quadratures():
    z, w = zwgj(5, 0.0, 0.0)
    assert abs(w.sum() - 2.0) < 1e-14
    assert abs(np.dot(w, z**8) - 2.0/9.0) < 1e-14
    z, w = gauss_legendre_lobatto(4)
    assert z[0] == -1.0 and z[-1] == 1.0
    assert abs(np.dot(w, z**4) - 2.0/5.0) < 1e-14


def test_inifile_semantics():
    cfg = Inifile('[a]\nX = 1 ; comment\ny = 2.5\n')
    assert cfg.get('a', 'X') == '1'
    assert cfg.getfloat('a', 'y') == 2.5
    assert cfg.getint('b', 'z', 7) == 7 and cfg.hasopt('b', 'z')
    with pytest.raises(Exception):
        cfg.get('a', 'missing')


def test_aosoa_layout_roundtrip():
    be = B200Backend(Inifile('[backend]\nprecision = double\n'),
                     device='cpu')
    rng = np.random.default_rng(0)
    a = rng.standard_normal((3, 5, 37))
    m = be.matrix(a.shape, a)
    np.testing.assert_array_equal(m.get(), a)
    nrow, ldim, _ = m.traits
    # frfs addressing: upt*ldim + ((e/32)*nvar + v)*32 + e%32
    flat = m.data.numpy()
    for (i, v, e) in [(0, 0, 0), (2, 4, 36), (1, 3, 31), (1, 2, 33)]:
        assert flat[i*ldim + ((e//32)*5 + v)*32 + e % 32] == a[i, v, e]
    assert ldim % 16 == 0 and ldim >= 5*64
