"""Build libgrimgpu.so in-tree for sm_100a (B200).

    python grim_20261007_b200/csrc/build.py [--verbose] [--ptxas-info]

The library lands next to the package (``grim_20261007_b200/libgrimgpu.so``), so it
travels with the source tree; nothing is installed into site-packages.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
SOURCES = ['grimgpu.cu']
HEADERS = ['common.cuh', 'hankel.cuh', 'fill2d.cuh', 'linalg.cuh', 'lu.cuh', 'tc_gemm.cuh', 'ozaki.cuh', 'dmma.cuh',
           'grouped.cuh', 'farblock.cuh', 'galerkin.cuh', 'pivot.cuh', 'condest.cuh', 'bor.cuh', 'noalloc.cu',
           'tslu.cuh', 'gepp_loop.cuh', 'modecond.cuh']
OUT = os.path.join(PKG, 'libgrimgpu.so')
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']


def nvcc_path():
    for cand in (os.environ.get('NVCC'), shutil.which('nvcc'), '/usr/local/cuda/bin/nvcc'):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError('nvcc not found')


def needs_build():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = SOURCES + HEADERS + ['../../include/grimgpu.h']
    for f in deps:
        p = os.path.join(HERE, f)
        if os.path.exists(p) and os.path.getmtime(p) > t:
            return True
    return False


def build(force=False, verbose=False, ptxas_info=False):
    if not force and not needs_build():
        return OUT
    cmd = [nvcc_path(), *ARCH, '-O3', '-lineinfo', '-std=c++17', '-Xcompiler', '-fPIC,-O2', '-shared',
           '--expt-relaxed-constexpr', '-o', OUT + '.tmp'] + [os.path.join(HERE, s) for s in SOURCES]
    if ptxas_info:
        cmd.insert(1, '-Xptxas=-v')
    if verbose:
        print(' '.join(cmd))
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError('nvcc failed building libgrimgpu.so')
    if verbose or ptxas_info:
        sys.stdout.write(res.stdout + res.stderr)
    os.replace(OUT + '.tmp', OUT)
    return OUT


if __name__ == '__main__':
    ap = argparse.ArgumentParser()
    ap.add_argument('--force', action='store_true')
    ap.add_argument('--verbose', action='store_true')
    ap.add_argument('--ptxas-info', action='store_true')
    a = ap.parse_args()
    print(build(force=True if (a.force or a.ptxas_info) else False, verbose=a.verbose, ptxas_info=a.ptxas_info))
