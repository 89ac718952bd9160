# -*- coding: utf-8 -*-
"""DGFS system: the solver-side operator API of frfs on the B200 library.

Keeps the interface of DGFSSystem (frfs/solvers/dgfs/system.py:17-231) that
the DGFS steppers and the ARS explicit stage call:

  collide(t, uinbank, foutbank)                       system.py:199-218
  updatebc(t, uinbank, foutbank, batch, varidx)       system.py:180-196
  rhs(t, uinbank, foutbank, batch, varidx)            system.py:140-177
  invmass(uinbank, foutbank)                          system.py:221-231

with the distribution banks addressed by register index
(``eles_scal_upts_inb_full``, system.py:127-136).  ``collide`` evaluates
Q(f) at every solution point in one persistent launch instead of a Python
loop of per-point launches; ``rhs`` and ``updatebc`` act on the velocity
slice [varidx, varidx + NvBatchSize) of the full banks in place (frfs copies
that slice through register banks first, system.py:140-196 with
integrators/base.py:166-214; the values are the same).  ``rk_stage`` fuses a
residual with the Runge-Kutta combination for the steppers.
"""

import ctypes as ct

import numpy as np

from frfs_b200 import _lib
from frfs_b200 import mesh as meshmod
from frfs_b200.elements import ElementGeometry
from frfs_b200.initcond import (MaxwellianSection, cylinder_wall_states,
                                initial_distribution)
from frfs_b200.scattering import DGFSScatteringModel, subclass_where
from frfs_b200.shapes import QuadShape
from frfs_b200.velocitymesh import DGFSVelocityMesh

c_int, c_ll, c_double, c_void_p = ct.c_int, ct.c_longlong, ct.c_double, \
    ct.c_void_p
c_dp, c_ip = ct.POINTER(ct.c_double), ct.POINTER(ct.c_int)


class DgParams(ct.Structure):
    """dgfs_dg_params (include/dgfs_b200.h)."""
    _fields_ = [('precision', c_int), ('ndims', c_int), ('nupts', c_int),
                ('nfpts', c_int), ('nvars', c_int), ('neles', c_int),
                ('soasz', c_int), ('ldim', c_ll), ('m0', c_dp),
                ('m132', c_dp), ('m3', c_dp), ('smats', c_dp),
                ('rcpdjac', c_dp), ('nrm', c_dp), ('mag', c_dp),
                ('partner', c_ip), ('cv', c_dp), ('cw', c_double),
                ('nbfpts', c_int), ('bkind', c_ip), ('bgroup', c_ip),
                ('bfpt', c_ip), ('bele', c_ip), ('ngroups', c_int),
                ('guw', c_dp), ('gfw', c_dp), ('grefl', c_ip),
                ('bwall', c_dp), ('m12', c_dp), ('nhalo', c_int),
                ('nsend', c_int), ('sfpt', c_ip), ('sele', c_ip)]


_lib.declare('dgfs_dg_create', c_int, [ct.POINTER(DgParams),
                                       ct.POINTER(c_void_p)])
_lib.declare('dgfs_dg_destroy', c_int, [c_void_p])
_lib.declare('dgfs_dg_interp', c_int, [c_void_p, c_void_p, c_int, c_int,
                                       c_void_p])
_lib.declare('dgfs_dg_updatebc', c_int, [c_void_p, c_int, c_int, c_int,
                                         c_void_p])
_lib.declare('dgfs_dg_rhs', c_int, [c_void_p, c_void_p, c_void_p, c_int,
                                    c_int, c_double, c_void_p, c_double,
                                    c_void_p, c_double, c_void_p, c_void_p])
_lib.declare('dgfs_dg_invmass', c_int, [c_void_p, c_void_p, c_void_p, c_int,
                                        c_int, c_void_p])
_lib.declare('dgfs_dg_pack', c_int, [c_void_p, c_void_p, c_void_p])
_lib.declare('dgfs_dg_set_halo', c_int, [c_void_p, c_void_p])
_lib.declare('dgfs_dg_num_variants', c_int, [c_void_p, c_ip])
_lib.declare('dgfs_dg_variant_info', c_int, [c_void_p, c_int, c_ip, c_ip,
                                             c_ip])
_lib.declare('dgfs_dg_select', c_int, [c_void_p, c_int])
_lib.declare('dgfs_dg_variant_tc', c_int, [c_void_p, c_int, c_ip])
_lib.declare('dgfs_dg_status', c_int, [c_void_p, c_void_p, c_ip])
_lib.declare('dgfs_dg_bcvals', c_int, [c_void_p, c_dp, c_int])
_lib.declare('dgfs_dg_fpts', c_int, [c_void_p, ct.POINTER(c_void_p),
                                     ct.POINTER(c_ll)])

# frfs boundary types (frfs/solvers/dgfs/inters.py) -> kernel kinds; the
# normal-shock inlet is the inlet with a zero velocity in its sign test
# (bcs/dgfs-inlet-normalshock.mako), the cylinder wall a diffuse wall with a
# wall state per boundary point
BC_KINDS = {'dgfs-wall-diffuse': 0, 'dgfs-inlet': 1, 'dgfs-outlet': 2,
            'dgfs-vanish': 3, 'dgfs-wall-specular': 4,
            'dgfs-inlet-normalshock': 1, 'dgfs-wall-diffuse-cyl': 5}


def _ptr(a, kind=c_dp):
    return a.ctypes.data_as(kind)


def specular_map(cv, n):
    """Reflected-velocity indices for a flat wall of unit normal n
    (frfs/solvers/dgfs/inters.py:258-275)."""
    n3 = np.zeros(3)
    n3[:len(n)] = n
    dot = n3 @ cv
    cr = cv - 2*dot[None, :]*n3[:, None]
    idx = np.empty(cv.shape[1], dtype=np.int32)
    for j in range(cv.shape[1]):
        idx[j] = np.argmin(np.sum((cr[:, j:j + 1] - cv)**2, axis=0))
    if not np.all(np.sort(idx) == np.arange(cv.shape[1])):
        raise ValueError('Non-unique specular map')
    return idx


class DGFSSystem:
    name = 'dgfs'

    def __init__(self, backend, cfg, mesh=None, nreg=3, initsoln=None,
                 sphdesign_paths=None, prank=0, halo_exchange=None):
        """``mesh`` in frfs's dictionary form, whole (keys ``*_p0``) or
        partitioned (``frfs_b200.partition.partition_mesh``), of which this
        system runs part ``prank``.  A part with faces shared with other
        parts exchanges their face values once per residual through
        ``halo_exchange(send, recv, nbrs, counts)`` (default:
        ``partition.exchange`` over torch.distributed, ranks = parts)."""
        self.backend = backend
        self.cfg = cfg
        self.vm = vm = DGFSVelocityMesh(backend, cfg, sphdesign_paths)
        self.mesh = mesh if mesh is not None else meshmod.from_config(cfg)
        self.prank = int(prank)
        self._sfx = f'_p{self.prank}'
        order = cfg.getint('solver', 'order')
        self.shape = sh = QuadShape(order)
        spt = self.mesh['spt_quad' + self._sfx]
        self.geo = geo = ElementGeometry(sh, spt)
        self.ndims = 2
        self.neles, self.nupts, self.nfpts = geo.neles, sh.nupts, sh.nfpts
        self.ele_types = ['quad']

        smn = cfg.get('scattering-model', 'type')
        self.sm = subclass_where(DGFSScatteringModel,
                                 scattering_model=smn)(backend, cfg, vm)

        V = vm.vsize()
        shape = (self.nupts, V, self.neles)
        ics = 'soln-ics'
        uniform = (cfg.get(ics, 'type', None) in ('maxwellian', 'bimaxwellian',
                                                  'bkw') and
                   not cfg.getfloat(ics, 'noise', 0.0))
        if initsoln is None and uniform:
            f0 = None
        elif initsoln is None:
            f0 = initial_distribution(cfg, vm, self.nupts, self.neles)
        elif isinstance(initsoln, dict):
            # a checkpoint (frfs's restart branch, system.py:79-112)
            from frfs_b200.checkpoint import restart_bank
            f0 = restart_bank(initsoln, cfg, V, self.mesh)
        else:
            f0 = np.asarray(initsoln).reshape(shape)
        mats = [backend.matrix(shape, f0 if i == 0 and f0 is not None
                               else None) for i in range(nreg)]
        if f0 is None:
            # a state uniform in space, filled on the device from its one
            # velocity vector (no host bank: the cylinder's full size is
            # 42 GB per FP32 bank, 84 GB in FP64 on the host)
            _fill_uniform(mats[0], initial_distribution(cfg, vm, 1, 1)[0, :,
                                                                        0])
        self.bank = backend.matrix_bank(mats)
        self.eles_scal_upts_inb_full = [self.bank]

        # time step for unit CFL (system.py:50-56)
        djac = geo.djac_at(sh.upts)
        self.unit_cfl_dt = float(np.sqrt(djac.min())/vm.L()/self.ndims)

        self.surrogate = None
        self.collide_hook = None
        self.halo_exchange = halo_exchange
        self._dg_shape = 0
        self._build_dg()

    # -- DG handle ----------------------------------------------------------
    def _build_dg(self):
        sh, geo, vm, cfg = self.shape, self.geo, self.vm, self.cfg
        E, F, V = self.neles, self.nfpts, vm.vsize()
        part = np.full((F, E), np.iinfo(np.int32).min, dtype=np.int64)
        lhs, rhs = self.mesh['con' + self._sfx]
        srtd = geo.srtd_face_fpts
        for l, r in zip(lhs, rhs):
            el, fl, er, fr = int(l['eidx']), int(l['fidx']), int(r['eidx']), \
                int(r['fidx'])
            for jl, jr in zip(srtd[fl][el], srtd[fr][er]):
                part[jl, el] = jr*E + er
                part[jr, er] = jl*E + el

        sfx = self._sfx
        bnames = sorted(k[5:-len(sfx)] for k in self.mesh
                        if k.startswith('bcon_') and k.endswith(sfx))
        bpts, guw, gfw, grefl, kinds = [], [], [], [], []
        self.bc_sections = {}
        for g, name in enumerate(bnames):
            sect = f'soln-bcs-{name}'
            btype = cfg.get(sect, 'type')
            if btype not in BC_KINDS:
                raise ValueError(f'unsupported boundary type {btype!r}')
            kinds.append(BC_KINDS[btype])
            if btype in ('dgfs-wall-diffuse', 'dgfs-inlet'):
                ms = MaxwellianSection(cfg, vm, sect)
                guw.append(ms.u)
                gfw.append(ms.values)
            elif btype == 'dgfs-inlet-normalshock':
                ms = MaxwellianSection(cfg, vm, sect)
                guw.append(np.zeros(3))
                gfw.append(ms.values)
            else:
                guw.append(np.zeros(3))
                gfw.append(np.zeros(V))
            recs = self.mesh[f'bcon_{name}{sfx}']
            for rec in recs:
                e, f = int(rec['eidx']), int(rec['fidx'])
                for j in srtd[f][e]:
                    bpts.append((g, int(j), e))
            if btype == 'dgfs-wall-specular':
                e0, f0 = int(recs[0]['eidx']), int(recs[0]['fidx'])
                n = geo.norm_pnorm_fpts[srtd[f0][e0][0], e0]
                for rec in recs:
                    e, f = int(rec['eidx']), int(rec['fidx'])
                    if not np.allclose(geo.norm_pnorm_fpts[srtd[f][e], e], n):
                        raise ValueError('specular walls must be flat')
                grefl.append(specular_map(vm.cv(), n))
            else:
                grefl.append(np.arange(V, dtype=np.int32))
            self.bc_sections[name] = (g, btype)
        bpts.sort(key=lambda x: (x[0], x[1], x[2]))
        nb = len(bpts)
        bkind = np.array([kinds[g] for g, _, _ in bpts], dtype=np.int32)
        bgroup = np.array([g for g, _, _ in bpts], dtype=np.int32)
        bfpt = np.array([j for _, j, _ in bpts], dtype=np.int32)
        bele = np.array([e for _, _, e in bpts], dtype=np.int32)
        for b, (g, j, e) in enumerate(bpts):
            part[j, e] = -(b + 1)
        # faces shared with other parts: halo row h of the received values
        from frfs_b200.partition import halo_rows
        nbrs, counts, hrows = halo_rows(self.mesh, self.prank, srtd)
        for h, (j, e) in enumerate(hrows):
            part[j, e] = -(len(bpts) + 1 + h)
        self.halo = (nbrs, counts) if hrows else None
        sfpt = np.array([j for j, _ in hrows] or [0], dtype=np.int32)
        sele = np.array([e for _, e in hrows] or [0], dtype=np.int32)
        # cylinder walls: the wall state at every boundary flux point
        bwall = np.ones((max(len(bpts), 1), 4))
        bwall[:, :3] = 0.0
        for name, (g, btype) in self.bc_sections.items():
            if btype != 'dgfs-wall-diffuse-cyl':
                continue
            idx = [b for b, (gb, _, _) in enumerate(bpts) if gb == g]
            xy = np.array([geo.plocfpts[j, e] for _, j, e in
                           (bpts[b] for b in idx)])
            bwall[idx] = cylinder_wall_states(cfg, vm, f'soln-bcs-{name}',
                                              xy[:, 0], xy[:, 1])
        if np.any(part == np.iinfo(np.int32).min):
            raise ValueError('mesh has flux points on no interface or '
                             'boundary')
        self.bpts = bpts

        d = lambda x: np.ascontiguousarray(x, dtype=np.float64)
        self._keep = keep = dict(
            m0=d(sh.opmat('M0')), m132=d(sh.opmat('M1 - M3*M2')),
            m3=d(sh.opmat('M3')), m12=d(sh.opmat('M12')),
            smats=d(geo.smat_at(sh.upts)),
            rcpdjac=d(geo.rcpdjac_at(sh.upts)),
            nrm=d(geo.norm_pnorm_fpts.transpose(0, 2, 1)),
            mag=d(geo.mag_pnorm_fpts),
            part=np.ascontiguousarray(part, dtype=np.int32),
            cv=d(vm.cv()), bkind=bkind, bgroup=bgroup, bfpt=bfpt, bele=bele,
            guw=d(np.array(guw).reshape(-1, 3)),
            gfw=d(np.array(gfw).reshape(-1, V)),
            grefl=np.ascontiguousarray(np.array(grefl).reshape(-1, V),
                                       dtype=np.int32),
            bwall=d(bwall))
        nrow, ldim, _ = self.bank[0].traits
        p = DgParams(
            precision=self.backend.precision, ndims=2, nupts=self.nupts,
            nfpts=F, nvars=V, neles=E, soasz=self.backend.soasz, ldim=ldim,
            m0=_ptr(keep['m0']), m132=_ptr(keep['m132']), m3=_ptr(keep['m3']),
            smats=_ptr(keep['smats']), rcpdjac=_ptr(keep['rcpdjac']),
            nrm=_ptr(keep['nrm']), mag=_ptr(keep['mag']),
            partner=_ptr(keep['part'], c_ip), cv=_ptr(keep['cv']),
            cw=vm.cw(), nbfpts=nb, bkind=_ptr(bkind, c_ip),
            bgroup=_ptr(bgroup, c_ip), bfpt=_ptr(bfpt, c_ip),
            bele=_ptr(bele, c_ip), ngroups=len(bnames),
            guw=_ptr(keep['guw']), gfw=_ptr(keep['gfw']),
            grefl=_ptr(keep['grefl'], c_ip), bwall=_ptr(keep['bwall']),
            m12=_ptr(keep['m12']), nhalo=len(hrows), nsend=len(hrows),
            sfpt=_ptr(sfpt, c_ip), sele=_ptr(sele, c_ip))
        keep['sfpt'], keep['sele'] = sfpt, sele
        h = c_void_p()
        lib = _lib.load()
        _lib.check(lib.dgfs_dg_create(ct.byref(p), ct.byref(h)),
                   'dgfs_dg_create')
        self._dg, self._lib = h, lib
        if self.halo is not None:
            import torch
            tdt = torch.float64 if self.backend.precision == 64 else \
                torch.float32
            self.halo_send = torch.zeros((len(hrows), V), dtype=tdt,
                                         device=self.backend.device)
            self.halo_recv = torch.zeros_like(self.halo_send)
            _lib.check(lib.dgfs_dg_set_halo(h, self.halo_recv.data_ptr()),
                       'dgfs_dg_set_halo')

    def __del__(self):
        h = getattr(self, '_dg', None)
        if h:
            self._lib.dgfs_dg_destroy(h)
            self._dg = None

    # -- frfs operator API ---------------------------------------------------
    def _range(self, batch, varidx):
        nvbs = self.vm.NvBatchSize()
        return int(varidx), nvbs

    def collide(self, t, uinbank, foutbank):
        """Q(f) at every solution point (system.py:199-218); through the
        attached learned surrogate (with its plain fallback) when
        ``self.surrogate`` is set.  ``collide_hook(fin, fout)``, when set,
        sees every (f, Q) pair (training-data collection)."""
        fin, fout = self.bank[uinbank], self.bank[foutbank]
        if self.surrogate is not None:
            self.surrogate.collide(fin, fout)
        else:
            self.sm.fs_all(fin, fout)
        if self.collide_hook is not None:
            self.collide_hook(fin, fout)

    @property
    def graph_key(self):
        """Part of a captured stage's key that changes with the collision
        path (plain, or a surrogate and its threshold)."""
        s = self.surrogate
        return None if s is None else (id(s), s.threshold)

    def updatebc(self, t, uinbank, foutbank, batch, varidx):
        """Face values of the slice and the diffuse-wall sums; the sums are
        reset on the slice that starts at velocity 0 (system.py:180-196)."""
        v0, nv = self._range(batch, varidx)
        u = self.bank[uinbank]
        s = self.backend.stream
        _lib.check(self._lib.dgfs_dg_interp(self._dg, u._as_parameter_, v0,
                                            nv, s), 'dgfs_dg_interp')
        if self.halo is not None and v0 + nv == self.vm.vsize():
            # face values of the shared faces to and from the neighbouring
            # parts, once the last velocity slice is interpolated
            # (inters.py:83-92: pack, send, recv; unpack is the residual's
            # direct read of the received rows)
            self.exchange_halo()
        _lib.check(self._lib.dgfs_dg_updatebc(self._dg, v0, nv,
                                              1 if v0 == 0 else 0, s),
                   'dgfs_dg_updatebc')

    def exchange_halo(self):
        """Pack this part's face values on shared faces and exchange them
        with the neighbouring parts (all velocities)."""
        _lib.check(self._lib.dgfs_dg_pack(self._dg, self.halo_send.data_ptr(),
                                          self.backend.stream), 'dgfs_dg_pack')
        nbrs, counts = self.halo
        fn = self.halo_exchange
        if fn is None:
            from frfs_b200.partition import exchange as fn
        fn(self.halo_send, self.halo_recv, nbrs, counts)

    def rhs(self, t, uinbank, foutbank, batch, varidx):
        """foutbank[slice] = -div F(uinbank[slice]) (system.py:140-177)."""
        v0, nv = self._range(batch, varidx)
        self.rk_stage(uinbank, foutbank, 0.0, None, 0.0, None, 1.0, None,
                      v0=v0, nv=nv)

    def rk_stage(self, uin, out, alpha, A, beta, B, gamma, C, v0=0, nv=None,
                 interp=True):
        """bank[out] = alpha bank[A] + beta bank[B] + gamma (L(bank[uin]) +
        bank[C]) on velocities [v0, v0 + nv) (bank indices or None)."""
        nv = self.vm.vsize() - v0 if nv is None else nv
        u = self.bank[uin]
        s = self.backend.stream
        if interp:
            _lib.check(self._lib.dgfs_dg_interp(self._dg, u._as_parameter_,
                                                v0, nv, s), 'dgfs_dg_interp')
        ptr = lambda i: None if i is None else self.bank[i]._as_parameter_
        _lib.check(self._lib.dgfs_dg_rhs(
            self._dg, u._as_parameter_, self.bank[out]._as_parameter_, v0,
            nv, alpha, ptr(A), beta, ptr(B), gamma, ptr(C), s),
            'dgfs_dg_rhs')

    def invmass(self, uinbank, foutbank):
        """bank[foutbank] = M12 bank[uinbank] at every solution point and
        velocity (system.py:221-231, elements.py:161-164)."""
        u, out = self.bank[uinbank], self.bank[foutbank]
        _lib.check(self._lib.dgfs_dg_invmass(
            self._dg, u._as_parameter_, out._as_parameter_, 0,
            self.vm.vsize(), self.backend.stream), 'dgfs_dg_invmass')

    # -- residual launch shapes (the autotuner's knob) -------------------------
    def dg_variants(self):
        """Compiled residual launch shapes: velocities per warp, whether
        the Runge-Kutta terms are loaded ahead of the flux work, CTAs per SM
        of the register budget, and whether the element-operator
        contraction runs on the tensor cores."""
        n = c_int()
        _lib.check(self._lib.dgfs_dg_num_variants(self._dg, ct.byref(n)),
                   'dgfs_dg_num_variants')
        out = []
        for i in range(n.value):
            v = [c_int() for _ in range(4)]
            _lib.check(self._lib.dgfs_dg_variant_info(
                self._dg, i, *[ct.byref(x) for x in v[:3]]),
                'dgfs_dg_variant_info')
            _lib.check(self._lib.dgfs_dg_variant_tc(
                self._dg, i, ct.byref(v[3])), 'dgfs_dg_variant_tc')
            out.append(dict(vpt=v[0].value, prefetch=v[1].value,
                            min_ctas_per_sm=v[2].value,
                            tensor_cores=bool(v[3].value)))
        return out

    def dg_status(self):
        """Raise if a bounded wait of the tensor-core residual ran out
        (synchronises the stream; clears the flag)."""
        flag = c_int()
        _lib.check(self._lib.dgfs_dg_status(self._dg, self.backend.stream,
                                            ct.byref(flag)),
                   'dgfs_dg_status')

    def select_dg(self, idx):
        _lib.check(self._lib.dgfs_dg_select(self._dg, int(idx)),
                   'dgfs_dg_select')
        self._dg_shape = int(idx)

    def autotune_dg(self, uin=0, out=1, reps=3):
        """Time every residual launch shape on a full Runge-Kutta stage of
        bank ``uin`` into bank ``out`` (overwritten: call before stepping)
        and keep the fastest; returns {shape index: ms}.  L2 is flushed
        (a 256 MiB write) before every timed launch, as a step finds it."""
        import torch
        dev = self.backend.device
        flush = torch.empty(64 << 20, dtype=torch.float32, device=dev)
        ms = {}
        # the flux-point values once (the same for every shape); each shape
        # then times its residual launch alone
        self.rk_stage(uin, out, 0.5, uin, 0.5, uin, 1e-4, uin, interp=True)
        for i in range(len(self.dg_variants())):
            self.select_dg(i)
            stage = lambda: self.rk_stage(uin, out, 0.5, uin, 0.5, uin, 1e-4,
                                          uin, interp=False)
            stage()
            torch.cuda.synchronize(dev)
            ev = [(torch.cuda.Event(enable_timing=True),
                   torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
            for e0, e1 in ev:
                flush.zero_()
                e0.record()
                stage()
                e1.record()
            torch.cuda.synchronize(dev)
            ms[i] = sum(e0.elapsed_time(e1) for e0, e1 in ev)/reps
        del flush
        self.dg_status()
        self.select_dg(min(ms, key=ms.get))
        return ms

    def moments(self, bankidx=None):
        """FP64 moments at every solution point of a bank, shape
        (nupts, neles, 14): rho, u(3), T, q(3), P(xx, xy, xz, yy, yz, zz)
        (frfs/plugins/dgfsmomwriterstd.py:154-214, nondimensional)."""
        return bank_moments(self.bank[self._active(bankidx)], self.vm,
                            self.backend)

    def _active(self, idx):
        return self.bank.active if idx is None else idx

    def bc_values(self):
        nb = len(self.bpts)
        buf = np.zeros(max(2*nb, 2))
        _lib.check(self._lib.dgfs_dg_bcvals(self._dg, _ptr(buf), buf.size),
                   'dgfs_dg_bcvals')
        return buf[:2*nb].reshape(nb, 2)

    def face_values(self):
        """Host copy of the face-value scratch (nfpts, V, neles)."""
        import torch
        p, ld = c_void_p(), c_ll()
        _lib.check(self._lib.dgfs_dg_fpts(self._dg, ct.byref(p),
                                          ct.byref(ld)), 'dgfs_dg_fpts')
        n = self.nfpts*ld.value
        view = _DeviceArray(p.value, n, '<f8' if self.backend.precision == 64
                            else '<f4')
        torch.cuda.synchronize(self.backend.device)
        buf = torch.as_tensor(view, device=self.backend.device)
        V, E = self.vm.vsize(), self.neles
        nblk = (E + 31)//32
        a = buf.view(self.nfpts, ld.value)[:, :nblk*32*V].cpu().numpy()
        a = a.reshape(self.nfpts, nblk, V, 32).transpose(0, 2, 1, 3)
        return a.reshape(self.nfpts, V, nblk*32)[:, :, :E]


def _fill_uniform(mat, f):
    """Every solution point of an AoSoA bank (nupts, V, neles) set to the
    velocity vector f (length V), padding lanes of the last element block
    left zero, on the device."""
    import torch
    nupts, V, neles = mat.ioshape
    nblk = (neles + 31)//32
    view = mat.view2d()[:, :nblk*V*32].view(nupts, nblk, V, 32)
    view.copy_(torch.as_tensor(np.asarray(f), dtype=view.dtype,
                               device=view.device)[None, None, :, None]
               .expand(nupts, nblk, V, 32))
    if neles % 32:
        view[:, nblk - 1, :, neles % 32:] = 0


def bank_moments(bank, vm, backend):
    """FP64 moments of a distribution bank on the device (dgfs_moments)."""
    import torch
    nupts, _, neles = bank.ioshape
    _, ldim, _ = bank.traits
    out = torch.empty(nupts*neles*14, dtype=torch.float64,
                      device=backend.device)
    _lib.check(_lib.load().dgfs_moments(
        backend.precision, bank._as_parameter_, nupts, neles, ldim, vm.Nv(),
        vm.L(), vm.cw(), out.data_ptr(), backend.stream), 'dgfs_moments')
    return out.view(nupts, neles, 14).cpu().numpy()


class _DeviceArray:
    """A device allocation described through __cuda_array_interface__."""

    def __init__(self, ptr, n, typestr):
        self.__cuda_array_interface__ = {'shape': (n,), 'typestr': typestr,
                                         'data': (ptr, False), 'version': 3}
