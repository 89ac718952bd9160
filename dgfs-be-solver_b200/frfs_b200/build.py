# -*- coding: utf-8 -*-
"""Build recipe for libdgfs_b200.so (sm_100a only).

Each ``csrc/*.cu`` translation unit is compiled with nvcc for
``arch=compute_100a,code=sm_100a`` and linked into one shared library placed
next to this file, where ``frfs_b200._lib`` loads it.  The CUDA runtime is
linked statically so the library carries no runtime dependency beyond the
driver.

    python -m frfs_b200.build          # from dgfs-be-solver_b200/
"""

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), 'csrc')
ROOT = os.path.dirname(os.path.dirname(HERE))
LIBNAME = 'libdgfs_b200.so'
LIBPATH = os.path.join(HERE, LIBNAME)
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
FLAGS = ['-std=c++17', '-O3', '-lineinfo', '-Xcompiler', '-fPIC',
         '-Xcompiler', '-fvisibility=hidden', '--expt-relaxed-constexpr']


def _nvcc():
    nv = shutil.which('nvcc') or '/usr/local/cuda/bin/nvcc'
    if not os.path.exists(nv):
        raise RuntimeError('nvcc not found; the CUDA toolkit is required')
    return nv


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC)
                  if f.endswith('.cu'))


def _needs_build(objdir):
    if not os.path.exists(LIBPATH):
        return True
    t = os.path.getmtime(LIBPATH)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(ROOT, 'include', 'dgfs_b200.h'))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, jobs=None):
    """Compile every csrc/*.cu for sm_100a and link libdgfs_b200.so."""
    objdir = os.path.join(os.path.dirname(HERE), '_build')
    if not force and not _needs_build(objdir):
        return LIBPATH
    os.makedirs(objdir, exist_ok=True)
    nvcc = _nvcc()

    def compile_one(src):
        obj = os.path.join(objdir, os.path.basename(src)[:-3] + '.o')
        cmd = [nvcc, *ARCH, *FLAGS, '-c', src, '-o', obj]
        if verbose:
            cmd.insert(1, '-Xptxas=-v')
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f'nvcc failed for {src}:\n{r.stderr}')
        if verbose and r.stderr:
            print(r.stderr, file=sys.stderr)
        return obj

    srcs = sources()
    with cf.ThreadPoolExecutor(jobs or min(8, len(srcs))) as ex:
        objs = list(ex.map(compile_one, srcs))
    tmp = LIBPATH + '.tmp'
    cmd = [nvcc, *ARCH, '-shared', '-o', tmp, *objs, '-cudart', 'static']
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f'link failed:\n{r.stderr}')
    os.replace(tmp, LIBPATH)
    return LIBPATH


if __name__ == '__main__':
    print(build(force='--force' in sys.argv, verbose='-v' in sys.argv))
