# -*- coding: utf-8 -*-
"""DGFS time steppers (frfs/integrators/std/steppers.py:20-225).

``StdEulerDGFSStepper`` ('dgfs-euler') and ``StdTVDRK2DGFSStepper``
('dgfs-tvd-rk2') advance the same stage values as frfs:

  Euler:  u^{n+1} = u^n + dt (L(u^n) + Q(u^n))
  RK2:    u1 = u^n + dt (L(u^n) + Q(u^n))
          u^{n+1} = u^n/2 + u1/2 + dt/2 (L(u1) + Q(u1))

where frfs loops over velocity batches, copies every batch through register
banks and applies axnpby kernels (steppers.py:122-225).  Here each stage is
one collision launch, one face interpolation, one boundary reduction and one
residual kernel whose epilogue performs the stage's linear combination; with
``[backend-b200] cuda-graphs = 1`` each stage is captured once as a CUDA
graph and replayed.

``step_reference_sequence`` keeps frfs's call order through the public
``collide / updatebc / rhs`` API and a separate combination per batch, for
integrators that drive the system themselves.
"""

import torch


class BaseDGFSStepper:
    stepper_name = None
    nregs = None

    def __init__(self, system, cfg):
        self.system = system
        self.cfg = cfg
        sect = 'solver-time-integrator'
        self.dt = cfg.getfloat(sect, 'dt')
        self.tcurr = cfg.getfloat(sect, 'tstart', 0.0)
        self.tend = cfg.getfloat(sect, 'tend', self.tcurr)
        self.nacptsteps = 0
        # a partitioned system exchanges face values with torch.distributed
        # point-to-point calls inside every stage; those stages run eagerly
        self.use_graphs = (cfg.getint('backend-b200', 'cuda-graphs', 0) == 1
                           and getattr(system, 'halo', None) is None)
        self._graphs = {}
        self._idxcurr = 0
        if len(system.bank) < self.nregs:
            raise ValueError(f'{self.stepper_name} needs {self.nregs} '
                             f'registers')

    @property
    def soln_bank(self):
        return self.system.bank[self._idxcurr]

    def _stage(self, key, fn):
        if not self.use_graphs:
            fn()
            return
        key = key + (self.system.graph_key,)
        g = self._graphs.get(key)
        if g is None:
            # First use: run the stage for real on a side stream (this is
            # the step's work), then capture it; capture executes nothing.
            dev = self.system.backend.device
            side = torch.cuda.Stream(device=dev)
            side.wait_stream(torch.cuda.current_stream(dev))
            with torch.cuda.stream(side):
                fn()
            torch.cuda.current_stream(dev).wait_stream(side)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                fn()
            self._graphs[key] = g
            return
        g.replay()

    def advance(self, nsteps):
        for _ in range(nsteps):
            self._idxcurr = self.step(self.tcurr, self.dt)
            self.tcurr += self.dt
            self.nacptsteps += 1
        return self._idxcurr


class StdEulerDGFSStepper(BaseDGFSStepper):
    stepper_name = 'dgfs-euler'
    nregs = 2

    def step(self, t, dt):
        s = self.system
        r0, r1 = (0, 1) if self._idxcurr == 0 else (1, 0)

        def stage():
            s.collide(t, r0, r1)
            s.updatebc(t, r0, r1, 0, 0)
            # r0 <- r0 + dt (L(r0) + Q(r0))   (steppers.py:66-98)
            s.rk_stage(r0, r1, 1.0, r0, 0.0, None, dt, r1, interp=False)
        self._stage(('euler', r0, dt), stage)
        return r1


class StdTVDRK2DGFSStepper(BaseDGFSStepper):
    stepper_name = 'dgfs-tvd-rk2'
    nregs = 3

    def step(self, t, dt):
        s = self.system
        r0, r1, r2 = 0, 1, 2
        if self._idxcurr != r0:
            r0, r1 = r1, r0

        def stage1():
            s.collide(t, r0, r1)
            s.updatebc(t, r0, r1, 0, 0)
            # r1 <- r0 + dt (L(r0) + Q(r0))   (steppers.py:157-178)
            s.rk_stage(r0, r1, 1.0, r0, 0.0, None, dt, r1, interp=False)

        def stage2():
            s.collide(t + dt, r1, r2)
            s.updatebc(t, r1, r2, 0, 0)
            # r0 <- r0/2 + r1/2 + dt/2 (L(r1) + Q(r1))   (steppers.py:197-221)
            s.rk_stage(r1, r0, 0.5, r0, 0.5, r1, 0.5*dt, r2, interp=False)

        self._stage(('rk2-1', r0, dt), stage1)
        self._stage(('rk2-2', r0, dt), stage2)
        return r0

    def step_reference_sequence(self, t, dt):
        """frfs's call order (steppers.py:122-225) through collide /
        updatebc / rhs, batch by batch."""
        s = self.system
        vm = s.vm
        nb, bs = vm.NvBatches(), vm.NvBatchSize()
        r0, r1, r2 = 0, 1, 2
        if self._idxcurr != r0:
            r0, r1 = r1, r0
        s.collide(t, r0, r1)
        for b in range(nb):
            s.updatebc(t, r0, r1, b, b*bs)
        for b in range(nb):
            s.rk_stage(r0, r1, 1.0, r0, 0.0, None, dt, r1, v0=b*bs, nv=bs)
        s.collide(t + dt, r1, r2)
        for b in range(nb):
            s.updatebc(t, r1, r2, b, b*bs)
        for b in range(nb):
            s.rk_stage(r1, r0, 0.5, r0, 0.5, r1, 0.5*dt, r2, v0=b*bs, nv=bs)
        return r0


STEPPERS = {c.stepper_name: c for c in (StdEulerDGFSStepper,
                                        StdTVDRK2DGFSStepper)}


def get_stepper(system, cfg):
    name = cfg.get('solver-time-integrator', 'scheme')
    if name not in STEPPERS:
        raise ValueError(f'unsupported scheme {name!r}')
    return STEPPERS[name](system, cfg)
