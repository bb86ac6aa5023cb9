"""Build the reference's own 2-D native far-block kernel as a checker (test infrastructure).

    python oracle/build_ref.py [reference_root]

Compiles ``tools/GHOST/ghost_backend/twod/assembly/native/far.c`` where it lies in the
reference tree, with the flags of the reference's own recipe
(``twod/assembly/native/build.py:96``: ``-O3 -std=c99 -ffp-contract=off``), into
``oracle/_ref/libghost_far_ref.so``.  The reference's build script itself is not run, and
no reference source is copied into this repository.  Only tests and ``bench.py``'s
reference leg load the result (as the checker and the timed reference CPU path of the
far-block pass); the product never does.  Without the reference tree (GPU machines) this
does nothing: the built library travels with the working tree instead.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, '_ref')
FAR_LIB = os.path.join(OUT_DIR, 'libghost_far_ref.so')
REL = os.path.join('tools', 'GHOST', 'ghost_backend', 'twod', 'assembly', 'native', 'far.c')


REFERENCE_ROOT = os.environ.get('GRIM_REFERENCE_ROOT', '/root/reference')


def build(reference_root=None):
    src = os.path.join(reference_root or REFERENCE_ROOT, REL)
    if not os.path.exists(src):
        return None
    cc = shutil.which('gcc') or shutil.which('cc')
    if cc is None:
        return None
    os.makedirs(OUT_DIR, exist_ok=True)
    tmp = FAR_LIB + '.tmp'
    subprocess.run([cc, '-O3', '-std=c99', '-ffp-contract=off', '-shared', '-fPIC', src, '-o', tmp, '-lm'],
                   check=True)
    os.replace(tmp, FAR_LIB)
    return FAR_LIB


if __name__ == '__main__':
    out = build(*(sys.argv[1:2] or []))
    print(out or 'reference tree not found: nothing built')
