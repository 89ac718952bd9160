# -*- coding: utf-8 -*-
"""B200 backend: device memory in frfs's matrix layout, streams, precision.

Matrices keep the layout contract of frfs/backends/base/types.py:9-102 so
that the same bank pointers can be handed to the C ABI:

* 2D ``(nrow, ncol)`` matrices are row-major;
* 3D ``(nrow, nvar, neles)`` and 4D ``(n0, n1, nvar, neles)`` matrices use
  the AoSoA(soasz=32) packing of frfs/backends/cuda/kernels/base.mako:4-6,
  value (i, v, e) at ``i*ldim + ((e/32)*nvar + v)*32 + e%32``;
* with the ``align`` tag the leading dimension is padded to 128 bytes
  (frfs/backends/cuda/base.py:49-52).

Device memory comes from PyTorch's caching allocator; streams are PyTorch
streams.  PyTorch is plumbing only: every numeric kernel lives in
libdgfs_b200.so.
"""

import numpy as np
import torch


class Matrix:
    def __init__(self, backend, ioshape, initval=None, tags=(), dtype=None):
        self.backend = backend
        self.tags = set(tags)
        self.dtype = np.dtype(dtype or backend.fpdtype)
        self.itemsize = self.dtype.itemsize
        ioshape = tuple(int(s) for s in ioshape)
        self.ioshape = ioshape

        ldmod = backend.alignb // self.itemsize if 'align' in self.tags else 1
        k = backend.soasz
        if len(ioshape) == 2:
            nrow, ncol = ioshape
            self.datashape = ioshape
        else:
            nvar, narr = ioshape[-2], ioshape[-1]
            nparr = narr - narr % -k
            nrow = ioshape[0] if len(ioshape) == 3 else ioshape[0]*ioshape[1]
            ncol = nvar*nparr
            self.datashape = ioshape[:-2] + (nparr // k, nvar, k)
        self.nrow, self.ncol = int(nrow), int(ncol)
        self.leaddim = self.ncol - (self.ncol % -ldmod)
        self.pitch = self.leaddim*self.itemsize
        self.nbytes = self.nrow*self.pitch
        self.traits = (self.nrow, self.leaddim, self.dtype)

        tdt = torch.float64 if self.dtype == np.float64 else torch.float32
        self.data = torch.zeros(self.nrow*self.leaddim, dtype=tdt,
                                device=backend.device)
        if initval is not None:
            self.set(initval)

    # ctypes integration, as CUDAMatrixBase._as_parameter_ in
    # frfs/backends/cuda/types.py:48-53
    @property
    def _as_parameter_(self):
        return self.data.data_ptr()

    def __index__(self):
        return self.data.data_ptr()

    def _pack(self, ary):
        ary = np.asarray(ary, dtype=self.dtype)
        if ary.ndim > 2:
            n, k = ary.shape[-1], self.backend.soasz
            ary = np.pad(ary, [(0, 0)]*(ary.ndim - 1) + [(0, -n % k)])
            ary = ary.reshape(ary.shape[:-1] + (-1, k)).swapaxes(-2, -3)
            ary = ary.reshape(self.nrow, self.ncol)
        return np.ascontiguousarray(ary)

    def _unpack(self, ary):
        if len(self.ioshape) > 2:
            ary = ary.reshape(self.datashape).swapaxes(-2, -3)
            ary = ary.reshape(self.ioshape[:-1] + (-1,))
            ary = ary[..., :self.ioshape[-1]]
        return ary

    def set(self, ary):
        if tuple(np.shape(ary)) != self.ioshape:
            raise ValueError(f'Invalid matrix shape {np.shape(ary)} != '
                             f'{self.ioshape}')
        buf = np.zeros((self.nrow, self.leaddim), dtype=self.dtype)
        buf[:, :self.ncol] = self._pack(ary)
        self.data.copy_(torch.from_numpy(buf.ravel()))

    def get(self):
        buf = self.data.view(self.nrow, self.leaddim)[:, :self.ncol]
        return self._unpack(buf.cpu().numpy())

    def view2d(self):
        """The (nrow, leaddim) storage as a torch tensor view."""
        return self.data.view(self.nrow, self.leaddim)


class MatrixBank:
    """A list of homogeneous matrices with an active index
    (frfs/backends/base/types.py:153-210)."""

    def __init__(self, mats, initbank=0):
        mats = list(mats)
        if any(m.traits != mats[0].traits for m in mats[1:]):
            raise ValueError('Matrices in a bank must be homogeneous')
        self._mats = mats
        self._curr_idx = initbank

    def __len__(self):
        return len(self._mats)

    def __getitem__(self, idx):
        return self._mats[idx]

    def __getattr__(self, attr):
        return getattr(self._mats[self._curr_idx], attr)

    @property
    def active(self):
        return self._curr_idx

    @active.setter
    def active(self, idx):
        self._curr_idx = idx


class B200Backend:
    name = 'b200'
    soasz = 32
    alignb = 128

    def __init__(self, cfg=None, device=None):
        prec = cfg.get('backend', 'precision', 'double') if cfg else 'double'
        if prec not in ('single', 'double'):
            raise ValueError('Invalid [backend] precision')
        self.fpdtype = np.float64 if prec == 'double' else np.float32
        self.precision = 64 if prec == 'double' else 32
        if device is None:
            device = torch.device('cuda', torch.cuda.current_device()) \
                if torch.cuda.is_available() else torch.device('cuda', 0)
        self.device = torch.device(device)
        self.cfg = cfg

    def matrix(self, ioshape, initval=None, tags=('align',), dtype=None):
        return Matrix(self, ioshape, initval, tags, dtype)

    def const_matrix(self, initval, tags=(), dtype=None):
        initval = np.asarray(initval)
        return Matrix(self, initval.shape, initval, tags, dtype)

    def matrix_bank(self, mats, initbank=0):
        return MatrixBank(mats, initbank)

    @property
    def stream(self):
        """The raw cudaStream_t of PyTorch's current stream."""
        return torch.cuda.current_stream(self.device).cuda_stream

    def synchronize(self):
        torch.cuda.synchronize(self.device)
