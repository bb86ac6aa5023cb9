"""Generate ``galerkin_near.npz``: the reference's own 2-D linear-Galerkin self and touching
element blocks on seeded straight elements.

Run in the build container (the reference tree is not present on GPU machines):

    python tests/golden/make_galerkin_near_golden.py /root/reference

The reference package is copied and its C kernels built as ``make_golden.py`` does.  It
records, for real wavenumbers:

* ``self``: single-layer self blocks ``_single_layer_block_linear`` (``twod/operators.py:1044``)
  of straight elements with |k L| from 0.05 to 60 -- the closed-form series (``:418``) up to
  |k L| = 8 and the composite sub-interval rule (``:980``) beyond;
* ``touch``: S and K' blocks of endpoint-touching element pairs by the graded two-triangle
  corner rule (``:629`` ``_integrate_linear_touching_duffy_sk_vectorized``), for collinear,
  right-angle, sharp and reflex corners, every combination of which end is shared, with the
  normal derivative on the source or on the observation element;
* ``ring`` / ``box``: on 60 random elements around a perturbed circle, the reference's
  adaptive-rule predicate (``twod/assembly/separation.py:67`` ``requires_adaptive``) for every
  non-adjacent pair closer than 4 element lengths, and the 16-point tensor S and K' blocks
  (``twod/operators.py:223`` ``_integrate_linear_pairs_box_sk_batched``) of the others, and the
  adaptive pairs' blocks by the reference's near-pair dispatcher (``:1080``
  ``_sk_blocks_near_linear``, whose bisection rule is ``:1172``), and the hypersingular blocks of
  the box pairs from their S blocks (``:1943`` ``_maue_blocks``);
* ``ring_S`` / ``ring_K``: the ring's whole node-based single-layer and observation-normal K'
  operators by the reference's own assembly (``twod/operators.py:1835``
  ``_assemble_linear_operator_matrices``: near routes, far pairs in one tile with its graded
  order, node scatter) at k = 30 and k = 4.
"""
from __future__ import annotations

import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)


def element(LE, name, p0, p1, index):
    p0, p1 = np.asarray(p0, float), np.asarray(p1, float)
    seg = p1 - p0
    length = float(np.hypot(*seg))
    tangent = seg / length
    normal = np.array([tangent[1], -tangent[0]])
    return LE(name=name, seg_type=2, ibc_flag=0, pos_mat=0, neg_mat=0, node_ids=(2 * index, 2 * index + 1), p0=p0,
              p1=p1, center=0.5 * (p0 + p1), tangent=tangent, normal=normal, length=length, panel_index=index)


def main(reference_root):
    sys.dont_write_bytecode = True
    from make_golden import _prepare
    _prepare(reference_root)
    from ghost_backend.twod import operators as O
    from ghost_backend.twod.geometry import LinearElement as LE
    rng = np.random.default_rng(20261205)
    out = {}
    # self blocks
    lengths, ks, blocks, ends = [], [], [], []
    for i, kl in enumerate((0.05, 0.7, 2.0, 5.5, 7.9, 8.5, 13.0, 21.0, 60.0)):
        length = float(rng.uniform(0.02, 0.3))
        k = kl / length
        p0 = rng.uniform(-1, 1, 2)
        ang = rng.uniform(0, 2 * math.pi)
        p1 = p0 + length * np.array([math.cos(ang), math.sin(ang)])
        e = element(LE, 'self', p0, p1, i)
        blocks.append(O._single_layer_block_linear(e, e, k))
        lengths.append(e.length)
        ks.append(k)
        ends.append(np.stack([p0, p1]))
    out.update(self_length=np.array(lengths), self_k=np.array(ks), self_s=np.array(blocks), self_ends=np.array(ends))
    # touching pairs: a corner at c, the observation element along direction a, the source
    # along direction b (angle between them = the corner's opening)
    rows = []
    for opening in (180.0, 90.0, 30.0, 170.0, 200.0, 330.0):
        for obs_start in (True, False):
            for src_start in (True, False):
                for obs_deriv in (False, True):
                    c = rng.uniform(-1, 1, 2)
                    base = rng.uniform(0, 2 * math.pi)
                    lo, ls = rng.uniform(0.05, 0.2, 2)
                    k = float(rng.uniform(2.0, 40.0))
                    da = np.array([math.cos(base), math.sin(base)])
                    db = np.array([math.cos(base + math.radians(opening)), math.sin(base + math.radians(opening))])
                    far_o, far_s = c + lo * da, c + ls * db
                    po = (c, far_o) if obs_start else (far_o, c)
                    ps = (c, far_s) if src_start else (far_s, c)
                    eo = element(LE, 'o', po[0], po[1], 0)
                    es = element(LE, 's', ps[0], ps[1], 1)
                    s_blk, k_blk = O._integrate_linear_touching_duffy_sk_vectorized(
                        eo, es, k, obs_deriv, (0.0, 1.0), (0.0, 1.0), obs_start, src_start, order=9)
                    rows.append((np.stack([po[0], po[1], ps[0], ps[1]]), k, obs_start, src_start, obs_deriv, s_blk,
                                 k_blk))
    out.update(touch_ends=np.array([r[0] for r in rows]), touch_k=np.array([r[1] for r in rows]),
               touch_obs_start=np.array([r[2] for r in rows]), touch_src_start=np.array([r[3] for r in rows]),
               touch_obs_deriv=np.array([r[4] for r in rows]), touch_s=np.array([r[5] for r in rows]),
               touch_kd=np.array([r[6] for r in rows]))
    # separated-near pairs: random straight elements around a perturbed circle; the
    # reference's own adaptive / box routing for every pair with centre distance < 4 L, and
    # its 16-point tensor blocks for the box pairs
    from ghost_backend.twod.assembly.separation import requires_adaptive
    n = 60
    t = np.sort(rng.uniform(0, 2 * math.pi, n))
    r = 0.5 * (1 + 0.15 * rng.standard_normal(n))
    pts = np.stack([r * np.cos(t), r * np.sin(t)], axis=1)
    import dataclasses
    elems = [dataclasses.replace(element(LE, 'e', pts[i], pts[(i + 1) % n], i), node_ids=(i, (i + 1) % n))
             for i in range(n)]
    pairs, adaptive = [], []
    for i in range(n):
        for j in range(n):
            if abs(i - j) in (0, 1, n - 1):
                continue
            a, b = elems[i], elems[j]
            if np.linalg.norm(a.center - b.center) < 4 * max(a.length, b.length):
                pairs.append((i, j))
                adaptive.append(bool(requires_adaptive(a, b)))
    pairs = np.array(pairs)
    adaptive = np.array(adaptive)
    box = pairs[~adaptive]
    k = 30.0
    s_box, k_box = O._integrate_linear_pairs_box_sk_batched(elems, box[:, 0], box[:, 1], k, False, 16)
    _s, k_box_obs = O._integrate_linear_pairs_box_sk_batched(elems, box[:, 0], box[:, 1], k, True, 16)
    out.update(ring_points=pts, ring_pairs=pairs, ring_adaptive=adaptive, ring_k=np.array(k), box_s=s_box,
               box_kd_src=k_box, box_kd_obs=k_box_obs)
    # the adaptive pairs through the reference's near-pair dispatcher (its bisection rule)
    close = pairs[adaptive]
    ad = [[O._sk_blocks_near_linear(elems[i], elems[j], k, deriv) for i, j in close] for deriv in (False, True)]
    out.update(adaptive_s=np.array([b[0] for b in ad[0]]), adaptive_kd_src=np.array([b[1] for b in ad[0]]),
               adaptive_kd_obs=np.array([b[1] for b in ad[1]]))
    # hypersingular blocks of the box pairs from their S blocks (the Maue identity)
    out['box_maue'] = O._maue_blocks(s_box, k, np.array([elems[i].normal for i in box[:, 0]]),
                                     np.array([elems[j].normal for j in box[:, 1]]),
                                     np.array([elems[i].length for i in box[:, 0]]),
                                     np.array([elems[j].length for j in box[:, 1]]))
    # the whole single-layer and K' (observation-normal) operators of the ring, node-based,
    # by the reference's own assembly (one tile: at most 192 elements)
    from ghost_backend.twod.geometry import LinearMesh, LinearNode
    mesh = LinearMesh(nodes=[LinearNode(xy=pts[i], key=(i, 0)) for i in range(n)], elements=elems)
    for kk, tag in ((30.0, 'k30'), (4.0, 'k4')):
        s_op, k_op = O._assemble_linear_operator_matrices(mesh, kk, True)
        out[f'ring_S_{tag}'] = np.asarray(s_op)
        out[f'ring_K_{tag}'] = np.asarray(k_op)
    np.savez_compressed(os.path.join(HERE, 'galerkin_near.npz'), **out)
    print('wrote galerkin_near.npz:', len(lengths), 'self blocks,', len(rows), 'touching pairs,', len(pairs),
          'near pairs (', int(adaptive.sum()), 'adaptive)')


if __name__ == '__main__':
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get('GRIM_REFERENCE_ROOT', '/root/reference'))
