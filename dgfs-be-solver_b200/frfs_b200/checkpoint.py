# -*- coding: utf-8 -*-
"""Distribution checkpoints and restart (frfs's distribution writer and
restart path).

frfs's writer plugin (frfs/plugins/dgfsdistwriterstd.py:41-66,
frfs/writers/native.py:86-186) stores the full distribution of every
element type as ``soln_<etype>_p<rank>`` with the run's ``config``, a
``stats`` file ([data] fields = f_0,...,f_{V-1}, prefix = soln, plus the
integrator's statistics) and the mesh's ``mesh_uuid``.  Restart
(frfs/__main__.py:228-242 -> frfs/solvers/dgfs/system.py:79-112) checks the
fields and interpolates the stored solution from the basis it was written
with onto the current solution points.  The same record is kept here in
one ``.npz`` file (h5py is not part of this package's dependencies); the
restart branch lives in ``restart_bank`` and is what ``DGFSSystem`` runs
when it is given a checkpoint as ``initsoln``.
"""

import hashlib

import numpy as np

from frfs_b200.inifile import Inifile
from frfs_b200.shapes import QuadShape


def _fields(V):
    return ','.join(f'f_{i}' for i in range(V))


def mesh_uuid(mesh):
    """A digest of the mesh arrays (frfs keeps the mesh file's uuid)."""
    h = hashlib.sha1()
    for k in sorted(mesh):
        a = np.ascontiguousarray(mesh[k])
        h.update(k.encode())
        h.update(a.tobytes())
    return h.hexdigest()


def solution_record(soln, cfg, tcurr, nacptsteps, mesh):
    """The checkpoint record of a solution array (nupts, V, neles)."""
    stats = Inifile()
    stats.set('data', 'fields', _fields(soln.shape[1]))
    stats.set('data', 'prefix', 'soln')
    stats.set('solver-time-integrator', 'tcurr', repr(float(tcurr)))
    stats.set('solver-time-integrator', 'nacptsteps', str(int(nacptsteps)))
    return {'soln_quad_p0': np.asarray(soln), 'config': cfg.tostr(),
            'stats': stats.tostr(), 'mesh_uuid': mesh_uuid(mesh)}


def write(path, system, stepper):
    """Checkpoint the stepper's current solution (one device-to-host copy
    of the bank)."""
    rec = solution_record(system.bank[stepper._idxcurr].get(), system.cfg,
                          stepper.tcurr, stepper.nacptsteps, system.mesh)
    np.savez(path, **rec)
    return path


def read(path):
    with np.load(path, allow_pickle=False) as z:
        return {k: (z[k] if k.startswith('soln_') else str(z[k]))
                for k in z.files}


def restart_bank(initsoln, cfg, V, mesh=None):
    """frfs/solvers/dgfs/system.py:79-112: the stored solution on the
    current solution points, shape (nupts, V, neles)."""
    solncfg = Inifile(initsoln['config'])
    solnsts = Inifile(initsoln['stats'])
    solnfields = solnsts.get('data', 'fields', '')
    if not solnfields or solnfields != _fields(V):
        raise RuntimeError('Invalid solution for system')
    if mesh is not None and initsoln.get('mesh_uuid') not in (
            None, mesh_uuid(mesh)):
        raise RuntimeError('solution was written on a different mesh')
    soln = np.asarray(initsoln['soln_quad_p0'], dtype=np.float64)
    solnb = QuadShape(solncfg.getint('solver', 'order'))
    curr = QuadShape(cfg.getint('solver', 'order'))
    if soln.shape[0] != solnb.nupts or soln.shape[1] != V:
        raise RuntimeError('stored solution does not match its config')
    if solnb.nupts == curr.nupts and np.allclose(solnb.upts, curr.upts):
        return soln  # same basis: the stored values, exactly
    interp = solnb.ubasis.nodal_basis_at(curr.upts)
    out = interp @ soln.reshape(solnb.nupts, -1)
    return out.reshape(curr.nupts, V, soln.shape[2])


def restart_time(initsoln):
    """(tcurr, nacptsteps) stored with the solution."""
    sts = Inifile(initsoln['stats'])
    return (sts.getfloat('solver-time-integrator', 'tcurr', 0.0),
            sts.getint('solver-time-integrator', 'nacptsteps', 0))
