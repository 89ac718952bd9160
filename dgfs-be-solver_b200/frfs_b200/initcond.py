# -*- coding: utf-8 -*-
"""Initial and boundary distributions (frfs/solvers/dgfs/initcond.py).

``maxwellian`` is frfs's DGFSMaxwellianInitCondition (initcond.py:39-116),
including its discrete-moment self-check; ``bkw`` is DGFSBKWInitCondition
(initcond.py:120-140).  ``bimaxwellian`` (two Maxwellians at +-ux, equal
weights, renormalised to the requested density) and the optional seeded
multiplicative noise of ``maxwellian`` (keys ``noise``, ``seed``) have no
counterpart in frfs; they describe the synthetic workloads.
"""

import numpy as np


def maxwellian_values(vm, rho, T, u):
    """Nondimensional Maxwellian on the velocity grid (initcond.py:62-64)."""
    u = np.asarray(u, dtype=np.float64).reshape(3, 1)
    return (rho/(np.pi*T)**1.5)*np.exp(-np.sum((vm.cv() - u)**2, axis=0)/T)


def _check_moments(vm, f, rho, T, u):
    """initcond.py:66-113: recompute rho, u, T on the grid; they must match
    the inputs (dimensional, absolute tolerance 1e-5)."""
    cv, cw = vm.cv(), vm.cw()
    s0 = np.sum(f)*cw
    s = [np.tensordot(f, cv[i], axes=(0, 0))*cw/s0 for i in range(3)]
    c = cv - np.array(s).reshape(3, 1)
    Tc = np.sum(f*np.sum(c*c, axis=0))*(2.0/3.0*cw)/s0
    ok = (np.allclose(rho*vm.rho0(), s0*vm.rho0(), atol=1e-5) and
          all(np.allclose(u[i]*vm.u0(), s[i]*vm.u0(), atol=1e-5)
              for i in range(3)) and
          np.allclose(T*vm.T0(), Tc*vm.T0(), atol=1e-5))
    if not ok:
        raise ValueError('Bulk properties not conserved! Check Nv, dev')


class MaxwellianSection:
    """rho, T, ux, uy, uz of a config section, nondimensionalised."""

    def __init__(self, cfg, vm, sect):
        self.rho = cfg.getfloat(sect, 'rho')/vm.rho0()
        self.T = cfg.getfloat(sect, 'T')/vm.T0()
        self.u = np.array([cfg.getfloat(sect, k)/vm.u0()
                           for k in ('ux', 'uy', 'uz')])
        self.values = maxwellian_values(vm, self.rho, self.T, self.u)
        _check_moments(vm, self.values, self.rho, self.T, self.u)


def initial_distribution(cfg, vm, nupts, neles, sect='soln-ics'):
    """Initial bank contents, shape (nupts, V, neles)."""
    kind = cfg.get(sect, 'type')
    V = vm.vsize()
    if kind == 'maxwellian':
        f = MaxwellianSection(cfg, vm, sect).values
        out = np.broadcast_to(f[None, :, None], (nupts, V, neles)).copy()
        noise = cfg.getfloat(sect, 'noise', 0.0)
        if noise:
            rng = np.random.default_rng(cfg.getint(sect, 'seed', 0))
            out *= 1.0 + noise*rng.standard_normal((nupts, V, neles))
        return out
    if kind == 'bimaxwellian':
        rho = cfg.getfloat(sect, 'rho')/vm.rho0()
        T = cfg.getfloat(sect, 'T')/vm.T0()
        u = np.array([cfg.getfloat(sect, k)/vm.u0()
                      for k in ('ux', 'uy', 'uz')])
        f = 0.5*(maxwellian_values(vm, 1.0, T, u) +
                 maxwellian_values(vm, 1.0, T, u*np.array([-1, 1, 1])))
        f *= rho/(np.sum(f)*vm.cw())
        return np.broadcast_to(f[None, :, None], (nupts, V, neles)).copy()
    if kind == 'bkw':
        t0 = cfg.getfloat(sect, 't0')
        K = 1.0 - np.exp(-t0/6.0)
        cSqr = np.sum(vm.cv()**2, axis=0)
        f = (1/(2*pow(2*np.pi*K, 1.5))*np.exp(-cSqr/(2.0*K)) *
             ((5*K - 3)/K + (1 - K)/(K*K)*cSqr))
        return np.broadcast_to(f[None, :, None], (nupts, V, neles)).copy()
    raise ValueError(f'unsupported initial condition type {kind!r}')


_EXPR_FUNCS = {'exp': np.exp, 'log': np.log, 'sqrt': np.sqrt, 'sin': np.sin,
               'cos': np.cos, 'tan': np.tan, 'tanh': np.tanh,
               'atan2': np.arctan2, 'pow': np.power, 'fabs': np.abs,
               'abs': np.abs, 'min': np.minimum, 'max': np.maximum}


def eval_point_expr(cfg, sect, key, x, y, z=None):
    """A boundary expression of frfs's config (``_exp_opts``,
    frfs/solvers/dgfs/inters.py:155-171: the [constants], x, y, z for the
    flux point's location, pi, abs) evaluated at the points (x, y[, z]).
    The expression passes Inifile.getexpr's character whitelist (no
    quotes, brackets or underscores), and is evaluated with no builtins."""
    expr = cfg.getexpr(sect, key)
    ns = dict(_EXPR_FUNCS)
    if 'constants' in cfg.sections():
        for k, v in cfg.items('constants').items():
            try:
                ns[k] = float(v)
            except (TypeError, ValueError):
                pass
    x = np.asarray(x, dtype=np.float64)
    ns.update(x=x, y=np.asarray(y, dtype=np.float64),
              z=np.zeros_like(x) if z is None else np.asarray(z, np.float64),
              pi=np.pi)
    val = eval(expr, {'__builtins__': {}}, ns)
    return np.broadcast_to(np.asarray(val, dtype=np.float64), x.shape).copy()


def cylinder_wall_states(cfg, vm, sect, x, y):
    """Nondimensional wall state (Ux, Uy, Uz, T) of a 'dgfs-wall-diffuse-cyl'
    boundary at the flux points (x, y): the section's ux, uy, uz, T
    expressions divided by u0 and T0 (inters.py:449-462); shape (n, 4)."""
    out = np.empty((len(np.atleast_1d(x)), 4))
    for i, k in enumerate(('ux', 'uy', 'uz')):
        out[:, i] = eval_point_expr(cfg, sect, k, x, y)/vm.u0()
    out[:, 3] = eval_point_expr(cfg, sect, 'T', x, y)/vm.T0()
    if not np.all(out[:, 3] > 0):
        raise ValueError(f'[{sect}] wall temperature must be positive')
    return out

