# -*- coding: utf-8 -*-
"""Generate golden fixtures by running pieces of the reference frfs package.

The reference (Ehsan-Roohi/DGFS-BE-Solver, package ``frfs``) cannot run as a
whole here: its kernels are Mako templates compiled by PyCUDA and its FFTs go
through cuFFT.  Its host-side numpy code does run once a few removed
Python/numpy names are shimmed and its GPU-only imports are replaced by empty
modules.  This script uses that to record, from the reference's own code:

* velocity mesh: L, cw, the 1D grid c0 and cv for small N
  (frfs/solvers/dgfs/velocitymesh.py:25-110);
* Gauss-Jacobi radial rule qz, qw (velocitymesh.py:112-126,
  frfs/quadratures.py:6-44);
* half-sphere spherical design sz, sw (velocitymesh.py:128-135,
  frfs/sphericaldesign/__init__.py:84-107) -- the tabulated Womersley designs
  used by the workloads are also copied, in their original text format, to
  the package's data folder ``frfs_b200/data/sphericaldesign/`` so that the
  solver, tests and benchmarks can load them on machines without the
  reference;
* VHS prefactor and gamma (frfs/solvers/dgfs/scattering.py:50-65);
* Maxwellian initial condition values (frfs/solvers/dgfs/initcond.py:39-116);
* quadrilateral FR operator matrices M0, M1, M2, M3, M1-M3*M2 and the point
  sets (frfs/shapes.py:83-166,243-289) for p = 1, 2, 3.

Run from the repository root, with DGFS_REFERENCE naming the directory of a
checkout of the reference::

    DGFS_REFERENCE=<path to the checkout> python tests/golden/make_golden.py
"""

import collections
import collections.abc
import configparser
import importlib.util
import os
import shutil
import sys
import types

import numpy as np

REF = os.environ.get('DGFS_REFERENCE')
HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, 'dgfs-be-solver_b200'))


def _install_shims():
    # Names removed from Python 3.10+/3.12 and numpy 2.x that frfs still uses
    collections.Iterable = collections.abc.Iterable
    collections.Sequence = collections.abc.Sequence
    np.float = float
    configparser.SafeConfigParser = configparser.ConfigParser

    def stub(name, **attrs):
        m = types.ModuleType(name)
        m.__dict__.update(attrs)
        sys.modules[name] = m
        return m

    sys.path.insert(0, REF)
    import frfs  # noqa: F401

    # GPU-only dependencies are replaced by empty modules; nothing below
    # calls into them.
    for n in ('pycuda', 'pycuda.gpuarray', 'pycuda.driver',
              'pycuda.compiler'):
        stub(n)
    sys.modules['pycuda'].gpuarray = sys.modules['pycuda.gpuarray']
    sys.modules['pycuda'].driver = sys.modules['pycuda.driver']
    sys.modules['pycuda'].compiler = sys.modules['pycuda.compiler']
    stub('frfs.template', DottedTemplateLookup=object)
    # Package __init__ files pull in MPI/h5py/plugins; load leaf modules only
    stub('frfs.solvers', __path__=[REF + '/frfs/solvers'])
    stub('frfs.solvers.dgfs', __path__=[REF + '/frfs/solvers/dgfs'])
    stub('frfs.solvers.dgfs.cufft', cufftPlan3d=None, cufftPlanMany=None,
         cufftExecD2Z=None, cufftExecZ2Z=None, CUFFT_D2Z=0, CUFFT_Z2Z=0,
         CUFFT_FORWARD=-1, CUFFT_INVERSE=1)
    stub('frfs.solvers.dgfs.cublas', CUDACUBLASKernels=object)
    stub('frfs.backends', __path__=[REF + '/frfs/backends'])
    stub('frfs.backends.cuda', __path__=[REF + '/frfs/backends/cuda'])
    stub('frfs.backends.cuda.provider', get_grid_for_block=None)


def _load(name):
    path = os.path.join(REF, *name.split('.')) + '.py'
    spec = importlib.util.spec_from_file_location(name, path)
    m = importlib.util.module_from_spec(spec)
    sys.modules[name] = m
    spec.loader.exec_module(m)
    return m


class _FakeBackend:
    soasz = 32
    alignb = 128

    def const_matrix(self, a, **kw):
        return a


def _maxwellian(icmod, cfg, vm, sect):
    ic = icmod.DGFSMaxwellianInitCondition(_FakeBackend(), cfg, vm, sect)
    return ic.get_init_vals()


def velocity_fixture(name, inistr, icmod, vmmod, scmod, Inifile, out,
                     with_ics=True):
    import contextlib
    import io

    cfg = Inifile(inistr)
    with contextlib.redirect_stdout(io.StringIO()):
        vm = vmmod.DGFSVelocityMesh(_FakeBackend(), cfg)
        sm = object.__new__(scmod.DGFSVHSGLLScatteringModel)
        sm.cfg, sm.vm, sm.backend = cfg, vm, _FakeBackend()
        sm.load_parameters()

        arrs = dict(
            ini=np.array(inistr), Nv=vm.Nv(), Nrho=vm.Nrho(), M=vm.M(),
            L=vm.L(), cw=vm.cw(), qz=vm.qz(), qw=vm.qw(), sz=vm.sz(),
            sw=vm.sw(), n0=vm.n0(), u0=vm.u0(), H0=vm.H0(), T0=vm.T0(),
            rho0=vm.rho0(), prefactor=sm._prefactor, gamma=sm._gamma,
            c0=np.unique(vm.cv()[0]),
        )
        if vm.vsize() <= 4096:
            arrs['cv'] = vm.cv()

        ics = cfg.get('soln-ics', 'type') if with_ics else None
        if ics == 'maxwellian':
            arrs['f0'] = _maxwellian(icmod, cfg, vm, 'soln-ics')
        elif ics == 'bimaxwellian':
            # Two frfs Maxwellians at +-ux: run the reference's own
            # Maxwellian initial condition on two derived sections
            ux = cfg.getfloat('soln-ics', 'ux')
            fs = []
            for s, sgn in (('ics-plus', 1.0), ('ics-minus', -1.0)):
                for k in ('rho', 'T', 'uy', 'uz'):
                    cfg.set(s, k, cfg.get('soln-ics', k))
                cfg.set(s, 'ux', repr(sgn*ux))
                fs.append(_maxwellian(icmod, cfg, vm, s))
            arrs['f0_plus'], arrs['f0_minus'] = fs

        for sect in cfg.sections():
            if with_ics and sect.startswith('soln-bcs-'):
                arrs['fw_' + sect[9:]] = _maxwellian(icmod, cfg, vm, sect)

    np.savez_compressed(os.path.join(out, f'ref_vm_{name}.npz'), **arrs)

    # Copy the spherical design table that this mesh loads
    npts = 2*vm.M()
    src = os.path.join(REF, 'frfs', 'sphericaldesign', 'symmetric')
    dst = os.path.join(ROOT, 'dgfs-be-solver_b200', 'frfs_b200', 'data',
                       'sphericaldesign')
    os.makedirs(dst, exist_ok=True)
    for f in os.listdir(src):
        if f.endswith(f'-m{npts:05d}.txt'):
            shutil.copyfile(os.path.join(src, f), os.path.join(dst, f))


def shapes_fixture(Inifile, out):
    import frfs.shapes as shapes

    for order in (1, 2, 3):
        cfg = Inifile(f"""
[solver]
order = {order}
[solver-elements-quad]
soln-pts = gauss-legendre
[solver-interfaces-line]
flux-pts = gauss-legendre
""")
        b = shapes.QuadShape(4, cfg)
        arrs = dict(
            upts=np.asarray(b.upts), fpts=np.asarray(b.fpts),
            norm_fpts=np.asarray(b.norm_fpts),
            nfacefpts=np.asarray(b.nfacefpts),
            M0=b.opmat('M0'), M1=b.opmat('M1'), M2=b.opmat('M2'),
            M3=b.opmat('M3'), M132=b.opmat('M1 - M3*M2'),
            M12=b.opmat('M12'),
        )
        np.savez_compressed(os.path.join(out, f'ref_shape_quad_p{order}.npz'),
                            **arrs)


def dg_fixture(Inifile, out):
    """Element geometry and interface pairing from frfs's own element code
    (frfs/solvers/base/elements.py:137-354, dgfs/elements.py:198-212) on a
    distorted 4x3 quadrilateral mesh, x-periodic, p = 2."""
    elmod = _load('frfs.solvers.base.elements')
    import frfs.shapes as shapes
    from frfs_b200 import mesh as mgen

    class _VM:
        def NvBatchSize(self):
            return 8

    for order, jitter in ((2, 0.2), (1, 0.15), (3, 0.1)):
        m = mgen.quad_box(4, 3, 0.0, 1.0, 0.0, 0.75, periodic_x=True,
                          jitter=jitter, seed=order)
        cfg = Inifile(f"""
[solver]
order = {order}
[solver-elements-quad]
soln-pts = gauss-legendre
[solver-interfaces-line]
flux-pts = gauss-legendre
""")

        class Eles(elmod.BaseElements):
            privarmap = {2: ['f_%d' % i for i in range(8)]}
            convarmap = privarmap
            _scratch_bufs = set()

            def set_backend(self, *a):
                pass

            @staticmethod
            def pri_to_con(p, c):
                return p

        ele = Eles(shapes.QuadShape, m['spt_quad_p0'], cfg)
        srtd = np.array([[list(x) for x in face]
                         for face in ele._srtd_face_fpts])
        arrs = dict(
            spt=m['spt_quad_p0'], con=m['con_p0'],
            bcon_bottom=m['bcon_bottom_p0'], bcon_top=m['bcon_top_p0'],
            smats_upts=ele.smat_at_np('upts'),
            rcpdjac_upts=ele.rcpdjac_at_np('upts'),
            djac_upts=ele.djac_at_np('upts'),
            ploc_upts=ele.ploc_at_np('upts'),
            plocfpts=ele.plocfpts,
            norm_pnorm_fpts=ele._norm_pnorm_fpts,
            mag_pnorm_fpts=ele._mag_pnorm_fpts,
            srtd_face_fpts=srtd,
        )
        np.savez_compressed(os.path.join(out, f'ref_dg_quad_p{order}.npz'),
                            **arrs)


def main():
    if not REF or not os.path.isdir(os.path.join(REF, 'frfs')):
        sys.exit('set DGFS_REFERENCE to the directory of a checkout of the '
                 'reference (it holds the frfs package)')
    _install_shims()
    vmmod = _load('frfs.solvers.dgfs.velocitymesh')
    icmod = _load('frfs.solvers.dgfs.initcond')
    scmod = _load('frfs.solvers.dgfs.scattering')
    from frfs.inifile import Inifile
    from frfs_b200 import workloads as wl

    # N=8 is too coarse for the reference's Maxwellian moment check, so the
    # small case records the velocity mesh and quadrature only
    small = wl.channel_n32(Nv=8, Nrho=4, M=6)
    cases = {
        'relax0d-n16': wl.relax0d_n16(),
        'couette-n24': wl.couette_n24(),
        'channel-n32': wl.channel_n32(),
        'small-n8': small,
    }
    for name, ini in cases.items():
        velocity_fixture(name, ini, icmod, vmmod, scmod, Inifile, HERE,
                         with_ics=(name != 'small-n8'))
    shapes_fixture(Inifile, HERE)
    import contextlib
    import io
    with contextlib.redirect_stdout(io.StringIO()):
        dg_fixture(Inifile, HERE)
    print('golden fixtures written to', HERE)


if __name__ == '__main__':
    main()
