"""Generate ``far_block.npz``: inputs and outputs of the reference's own far-field
Galerkin block quadrature (``twod/assembly/native/far.c:193`` ``ghost_far_block``).

Run in the build container (the reference tree is not present on GPU machines):

    python oracle/build_ref.py            # the reference's far.c -> oracle/_ref/libghost_far_ref.so
    python tests/golden/make_far_golden.py /root/reference

The kernel table is the reference's own (``twod/assembly/kernels.py:337`` ``KernelTable``,
imported from the reference tree without writing into it: its ``bounds`` and
``normalized_power`` are what ``far.py:184-249`` passes to the native kernel); the element
geometry is seeded: random straight elements of a perturbed circle, Gauss-Legendre points
(``numpy.polynomial.legendre.leggauss``, as ``twod/operators.py:3320``), linear (width 2)
and quadratic (width 3) Lagrange bases at the points, a far mask from the element-centre
distance, and a few source elements beyond the table's upper distance so that the
large-argument branch is exercised.  For each case the reference library is called through
ctypes exactly as ``far.py:221-234`` calls it.
"""
from __future__ import annotations

import ctypes as ct
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def reference_far(lib, obs_pts, src_pts, qw, phi, on, sn, far, ond, want_s, want_k, mirrored, k, bounds, power):
    fun = lib.ghost_far_block
    p = ct.c_void_p
    fun.argtypes = [ct.c_int64, ct.c_int64, ct.c_int, ct.c_int] + [p] * 7 + [ct.c_int] * 4 + [ct.c_double] * 2 + \
                   [ct.c_int, p, ct.c_int, p, p, p, p]
    fun.restype = ct.c_int
    mb, q = obs_pts.shape[:2]
    nb, width = src_pts.shape[0], phi.shape[1]
    bufs = [np.zeros((width * width, mb, nb), complex) if w else None
            for w in (want_s, want_k, want_k and mirrored)]
    status = fun(mb, nb, q, width, obs_pts.ctypes.data, src_pts.ctypes.data, qw.ctypes.data, phi.ctypes.data,
                 on.ctypes.data, sn.ctypes.data, far.ctypes.data, ond, want_s, want_k, mirrored, k.real, k.imag,
                 len(bounds) - 1, bounds.ctypes.data, power.shape[1] - 1, power.ctypes.data,
                 *(None if b is None else b.ctypes.data for b in bufs))
    return status, bufs


def geometry(rng, count, radius, q, width, far_out=0, far_distance=0.0):
    """Straight elements of a perturbed circle; returns obs/src points, weights, basis,
    outward normals and centres.  The last `far_out` source elements are moved out by
    `far_distance`."""
    t = np.sort(rng.uniform(0, 2 * np.pi, count + 1))[:count]
    t = np.r_[t, t[0] + 2 * np.pi]
    rr = radius * (1 + 0.1 * rng.standard_normal(count + 1))
    rr[-1] = rr[0]
    pts = np.stack([rr * np.cos(t), rr * np.sin(t)], -1)
    a, b = pts[:-1], pts[1:]
    x, w = np.polynomial.legendre.leggauss(q)
    s = (x + 1) / 2
    p = a[:, None, :] * (1 - s)[None, :, None] + b[:, None, :] * s[None, :, None]
    tan = b - a
    length = np.linalg.norm(tan, axis=1)
    normal = np.stack([tan[:, 1], -tan[:, 0]], -1) / length[:, None]
    if width == 2:
        phi = np.stack([(1 - x) / 2, (1 + x) / 2], -1)
    else:
        phi = np.stack([x * (x - 1) / 2, 1 - x * x, x * (x + 1) / 2], -1)
    src = p.copy()
    if far_out:
        src[-far_out:] += far_distance * normal[-far_out:, None, :]
    return p, src, w * 0.5, phi, normal, (a + b) / 2, length


def main(reference_root):
    sys.dont_write_bytecode = True
    sys.path.insert(0, os.path.join(reference_root, 'tools', 'GHOST'))
    from ghost_backend.twod.assembly.kernels import KernelTable
    lib_path = os.path.join(ROOT, 'oracle', '_ref', 'libghost_far_ref.so')
    if not os.path.exists(lib_path):
        raise SystemExit('build the checker first: python oracle/build_ref.py')
    lib = ct.CDLL(lib_path)
    rng = np.random.default_rng(20261203)
    out = {}
    cases = [('w2', 40.0 + 0j, 2, 5), ('w3', 25.0 - 0.4j, 3, 4)]
    for name, k, width, q in cases:
        upper = 1.6
        table = KernelTable(k, upper)
        bounds = np.ascontiguousarray(table.bounds, np.float64)
        power = np.ascontiguousarray(table.normalized_power, np.complex128)
        obs, _src, qw, phi, on, centre, length = geometry(rng, 18, 0.5, q, width)
        obs2, src, _qw, _phi, sn, centre_s, _l = geometry(rng, 16, 0.5, q, width, far_out=4, far_distance=2.0)
        dcent = np.linalg.norm(centre[:, None, :] - (src.mean(axis=1))[None, :, :], axis=-1)
        far = (dcent > 2.5 * np.median(length)).astype(np.uint8)
        far[3, 5] = 0
        out[f'{name}_k'] = np.array(k)
        out[f'{name}_bounds'] = bounds
        out[f'{name}_power'] = power
        out[f'{name}_upper'] = np.array(upper)
        for key, val in (('obs_pts', obs), ('src_pts', src), ('qw', qw), ('phi', phi), ('obs_norm', on),
                         ('src_norm', sn), ('far', far)):
            out[f'{name}_{key}'] = np.ascontiguousarray(val)
        for ond in (0, 1):
            status, (s, kk, kt) = reference_far(lib, *(np.ascontiguousarray(out[f'{name}_{key}']) for key in
                                                       ('obs_pts', 'src_pts', 'qw', 'phi', 'obs_norm', 'src_norm',
                                                        'far')), ond, 1, 1, 1, k, bounds, power)
            assert status == 0, status
            out[f'{name}_ond{ond}_s'] = s
            out[f'{name}_ond{ond}_k'] = kk
            out[f'{name}_ond{ond}_kt'] = kt
    np.savez_compressed(os.path.join(HERE, 'far_block.npz'), **out)
    print('wrote far_block.npz', {k: v.shape for k, v in out.items() if k.endswith('_s') or k.endswith('bounds')})


if __name__ == '__main__':
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get('GRIM_REFERENCE_ROOT', '/root/reference'))
