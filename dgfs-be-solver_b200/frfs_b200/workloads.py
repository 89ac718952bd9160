# -*- coding: utf-8 -*-
"""Named DGFS workloads as frfs-style ``.ini`` strings.

Each workload is a complete configuration in the same sections and keys that
frfs reads (``[constants]``, ``[non-dim]``, ``[velocity-mesh]``,
``[spherical-design-rule]``, ``[scattering-model]``, ``[solver]``,
``[soln-ics]``, ``[soln-bcs-*]``), plus the mesh description this package
generates itself (``[mesh]``).  The key names follow
frfs/solvers/dgfs/velocitymesh.py:25-135, frfs/solvers/dgfs/scattering.py:50-65,
frfs/solvers/dgfs/initcond.py:39-116 and frfs/solvers/dgfs/inters.py:175-229.

Workloads
---------
relax0d-n16   single point, N=16, Nrho=8, M=6, VHS omega=0.5, L=5 (hard
              sphere 0D relaxation of two Maxwellians at u=(+-1.5,0,0)).
couette-n24   64x1 quadrilateral strip, p=2, N=24, Nrho=12, M=16, omega=0.81,
              diffuse walls at x=+-1/2 moving at uy=+-0.5 (nondimensional),
              y-periodic; dt = 1e-4: the p=2 FR-DG operator with SSP-RK2 is
              stable for |c| dt / h <= 0.056 at the corner velocity
              |cx| = |cy| = 5.27 on this strip (eigenvalues of the operator);
              1e-4 gives 0.034.  M=16 replaces the requested M=12: the tabulated
              symmetric designs hold 2M in {2,6,12,32,48,70,...} points only.
cylinder-n32  quadrilateral O-grid around a cylinder, p=3, N=32, Nrho=16,
              M=24, Mach-2 inflow, diffuse cylinder wall (cylinder_n32).
channel-n32   48x24 quadrilaterals, p=2 (10368 points), N=32, Nrho=16, M=24,
              x-periodic, diffuse walls at y=+-1/4, Maxwellian times
              (1 + 0.01 xi) with xi ~ N(0,1) per velocity node and point;
              dt = 1e-4 (|c| dt / h = 0.023 at the corner velocity; the
              p=2 FR-DG operator with SSP-RK2 on a 2D periodic box is
              stable up to 0.036).
"""

import numpy as np

# Argon (frfs examples use the same reference gas)
_MOLAR_MASS = 39.96e-3
_R0 = 8.3144598


def _u0(T0=273.0, molarMass0=_MOLAR_MASS):
    return float(np.sqrt(2*_R0/molarMass0*T0))


_BASE = """
[backend]
precision = {precision}

[constants]
Nv = {Nv}
NvBatchSize = {NvBatchSize}
Nrho = {Nrho}

[non-dim]
T0 = 273.0
H0 = {H0}
rho0 = {rho0}
molarMass0 = {molarMass0}

[velocity-mesh]
cmax = {cmax}
Tmax = 273.0
dev = {dev}
quad-rule = jacobi
quad-rule-alpha = 0
quad-rule-beta = 0

[spherical-design-rule]
ssrule = womersley
M = {M}

[scattering-model]
type = vhs-gll
omega = {omega}
dRef = 4.17e-10
Tref = 273.0

[solver]
system = dgfs
order = {order}

[solver-time-integrator]
scheme = dgfs-tvd-rk2
controller = none
tstart = 0.0
tend = {tend}
dt = {dt}

[solver-interfaces]
riemann-solver = rusanov

[solver-interfaces-line]
flux-pts = gauss-legendre

[solver-elements-quad]
soln-pts = gauss-legendre
"""


def relax0d_n16(precision='double'):
    """Space-homogeneous relaxation at one point: N = 16, Nrho = 8, M = 6,
    FP64, from the bimodal state of two Maxwellians at u = +-1.5."""
    u0 = _u0()
    ini = _BASE.format(precision=precision, Nv=16, NvBatchSize=4096, Nrho=8,
                       H0=1e-3, rho0=1.5e-3, molarMass0=_MOLAR_MASS,
                       cmax=0.0, dev=5.0, M=6, omega=0.5, order=2,
                       tend=0.5, dt=0.01)
    ini += f"""
[soln-ics]
type = bimaxwellian
rho = 1.5e-3
T = 273.0
ux = {1.5*u0!r}
uy = 0.0
uz = 0.0
"""
    return ini


def couette_n24(precision='double', M=16, nele=64, copies=1):
    """1D/3V Couette slab as a 64x1 quad strip (576 points at p = 2,
    N = 24, Nrho = 12, M = 16, walls at U = +-0.5).
    ``copies`` > 1 widens the slab to that many slab widths (nele elements
    each, the same element size) for weak scaling over partitions."""
    u0 = _u0()
    ini = _BASE.format(precision=precision, Nv=24, NvBatchSize=13824,
                       Nrho=12, H0=1e-3, rho0=1.5e-3,
                       molarMass0=_MOLAR_MASS, cmax=repr(0.5*u0), dev=5.0,
                       M=M, omega=0.81, order=2, tend=0.02, dt=1e-4)
    ini += f"""
[mesh]
type = quad-strip
nx = {nele*copies}
ny = 1
xlo = {-0.5*copies!r}
xhi = {0.5*copies!r}
ylo = 0.0
yhi = {1.0/nele!r}
periodic-y = 1

[soln-ics]
type = maxwellian
rho = 1.5e-3
T = 273.0
ux = 0.0
uy = 0.0
uz = 0.0

[soln-bcs-left]
type = dgfs-wall-diffuse
rho = 1.5e-3
T = 273.0
ux = 0.0
uy = {-0.5*u0!r}
uz = 0.0

[soln-bcs-right]
type = dgfs-wall-diffuse
rho = 1.5e-3
T = 273.0
ux = 0.0
uy = {0.5*u0!r}
uz = 0.0
"""
    return ini


def channel_n32(precision='double', nx=48, ny=24, Nv=32, Nrho=16, M=24,
                copies=1):
    """2D/3V channel on 48x24 quads (10,368 points at p = 2, N = 32).  ``copies``
    > 1 lengthens the periodic channel to that many channel lengths (nx
    elements each) for weak scaling over partitions."""
    ini = _BASE.format(precision=precision, Nv=Nv, NvBatchSize=Nv**3,
                       Nrho=Nrho, H0=1e-3, rho0=1.5e-3,
                       molarMass0=_MOLAR_MASS, cmax=0.0, dev=5.0, M=M,
                       omega=0.81, order=2, tend=0.02, dt=1e-4)
    ini += f"""
[mesh]
type = quad-box
nx = {nx*copies}
ny = {ny}
xlo = {-0.5*copies!r}
xhi = {0.5*copies!r}
ylo = -0.25
yhi = 0.25
periodic-x = 1

[soln-ics]
type = maxwellian
rho = 1.5e-3
T = 273.0
ux = 0.0
uy = 0.0
uz = 0.0
noise = 0.01
seed = 0

[soln-bcs-bottom]
type = dgfs-wall-diffuse
rho = 1.5e-3
T = 273.0
ux = 0.0
uy = 0.0
uz = 0.0

[soln-bcs-top]
type = dgfs-wall-diffuse
rho = 1.5e-3
T = 273.0
ux = 0.0
uy = 0.0
uz = 0.0
"""
    return ini


def _ogrid_hmin(ntheta, nr, stretch, r_in=0.5, r_out=4.0):
    """sqrt(area) of the innermost O-grid element: the first radial size
    times the arc length at the cylinder."""
    w = stretch**np.arange(nr)
    dr0 = (r_out - r_in)*w[0]/np.sum(w)
    return float(np.sqrt(dr0*r_in*2*np.pi/ntheta))


def cylinder_n32(precision='single', ntheta=40, nr=16, order=3, Nv=32,
                 Nrho=16, M=24, mach=2.0, dt=None, tend=0.01):
    """Cylinder in a Mach-2 crossflow on a
    quadrilateral O-grid, p=3, N=32, Nrho=16, M=24 (M=32 has no tabulated
    symmetric design; the 48-point rule of M=24 is the nearest).  Cylinder
    of radius 0.5 with a diffuse isothermal wall (``dgfs-wall-diffuse-cyl``,
    wall at rest, T_w = T_inf), far field at radius 4: Maxwellian inflow
    on the upstream half, outflow on the downstream half; uniform freestream
    initial state.  Speeds: the freestream speed is mach * sqrt(5/6) u0
    (sound speed of a monatomic gas at T0 in units of u0 = sqrt(2 R T0)).

    Full size is ntheta x nr ~ 20 000 elements (ntheta=160, nr=125: 320 000
    points, 42 GB per FP32 bank); the default, 40 x 16 = 640 elements
    (10 240 points), has the channel's point count.  The radial sizes grow
    geometrically by 1.15 per element up to nr = 16; finer grids keep the
    default's total growth of 1.15**15 (8.1) from the cylinder to the far
    field (stretch 1.017 at nr = 125).
    dt = 2e-4 on the default grid gives |c| dt / h = 0.023 on the smallest
    element (h = sqrt(area) = 0.070) at the corner speed of the velocity
    box (|c| = 8.2); the p=3 FR-DG operator with SSP-RK2 on O-grids is
    stable up to 0.055 (eigenvalues of the operator on 12x2 and 16x3
    O-grids).  dt = None scales 2e-4 by the smallest element's h against
    the default grid's, which keeps |c| dt / h = 0.023 at every size."""
    stretch = 1.15**min(1.0, 15.0/max(nr - 1, 1))
    if dt is None:
        dt = 2e-4*_ogrid_hmin(ntheta, nr, stretch)/_ogrid_hmin(40, 16, 1.15)
    u0 = _u0()
    uinf = float(mach*np.sqrt(5.0/6.0)*u0)
    ini = _BASE.format(precision=precision, Nv=Nv, NvBatchSize=Nv**3,
                       Nrho=Nrho, H0=1e-3, rho0=1.5e-3,
                       molarMass0=_MOLAR_MASS, cmax=0.0, dev=6.0, M=M,
                       omega=0.81, order=order, tend=tend, dt=dt)
    ini += f"""
[mesh]
type = quad-ogrid
ntheta = {ntheta}
nr = {nr}
r-in = 0.5
r-out = 4.0
stretch = {stretch!r}

[soln-ics]
type = maxwellian
rho = 1.5e-3
T = 273.0
ux = {uinf!r}
uy = 0.0
uz = 0.0

[soln-bcs-cylinder]
type = dgfs-wall-diffuse-cyl
ux = 0.0
uy = 0.0
uz = 0.0
T = 273.0

[soln-bcs-inflow]
type = dgfs-inlet
rho = 1.5e-3
T = 273.0
ux = {uinf!r}
uy = 0.0
uz = 0.0

[soln-bcs-outflow]
type = dgfs-outlet
"""
    return ini


WORKLOADS = {
    'relax0d-n16': relax0d_n16,
    'couette-n24': couette_n24,
    'channel-n32': channel_n32,
    'cylinder-n32': cylinder_n32,
}


def mixture_n24(precision='single', Nv=24, Nrho=12, M=32, Mpre=32):
    """Binary argon-krypton mixture for frfs's dgfsbi VSS operator
    (frfs/solvers/dgfsbi/velocitymesh.py:27-151, scattering.py:44-330):
    N=24, Nrho=12, the 32-point full-sphere design for the directions and
    for the precomputation of the direction-dependent gain kernel, and
    Bird's VSS parameters (Ar: alpha 1.40, omega 0.81, d 4.11e-10 m; Kr:
    alpha 1.32, omega 0.80, d 4.76e-10 m; the unlike pair takes the
    means).  The collision operator alone: no mesh, no solver section."""
    gas = {'0': (1.40, 0.81, 4.11e-10), '1': (1.32, 0.80, 4.76e-10)}
    lines = []
    for p in '01':
        for q in '01':
            a = 0.5*(gas[p][0] + gas[q][0])
            w = 0.5*(gas[p][1] + gas[q][1])
            d = 0.5*(gas[p][2] + gas[q][2])
            lines.append(f'alpha{p}{q} = {a!r}\nomega{p}{q} = {w!r}\n'
                         f'dRef{p}{q} = {d!r}\nTref{p}{q} = 273.0')
    sm = '\n'.join(lines)
    return f"""
[backend]
precision = {precision}

[constants]
Nv = {Nv}
Nrho = {Nrho}

[non-dim]
T0 = 273.0
H0 = 1e-3
rho0 = 1.5e-3
molarMass0 = {_MOLAR_MASS!r}

[velocity-mesh]
cmax = 0.0
Tmax = 273.0
dev = 5.0
molarMass1 = {_MOLAR_MASS!r}
molarMass2 = 83.8e-3

[spherical-design-rule]
ssrule = womersley
M = {M}

[scattering-model]
type = vss-gll
ssrulepre = womersley
Mpre = {Mpre}
{sm}
"""


# collision-operator-only workloads (bench.py --mode collide)
MIXTURES = {
    'mixture-n24': mixture_n24,
}
