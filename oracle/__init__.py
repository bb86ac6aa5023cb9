"""CPU oracle for the GPU RCS solve path.

THIS PACKAGE IS TEST INFRASTRUCTURE.  Only ``tests/``, ``__graft_entry__.smoke()``
and the ``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import it,
and only as the checker (or as the timed CPU stand-in for the reference's own CPU
solve).  The product package ``grim_20261007_b200`` never imports it.

Contents
--------
``pulse2d``  FP64 NumPy/SciPy restatement of the pulse-basis, point-matched 2-D
             TM EFIE and TE MFIE that the GPU kernels implement (fill, plane-wave
             excitation, monostatic far-field projection, sigma_2D).
``mie``      Analytic PEC cylinder / sphere series, restated from the reference's
             ``ghost_backend/validation/cylinder.py:37-72`` and ``sphere.py:196``.
``bor``      FP64 restatement of the body-of-revolution per-mode EFIE/MFIE/CFIE
             that the GPU BoR path implements.

Pinning
-------
* ``mie`` is pinned against the reference's own Mie functions
  (``tests/golden/mie_cylinder.npz``, generated by ``tests/golden/make_golden.py``
  from the reference in the build container).
* ``pulse2d`` is pinned physically: against ``mie`` at the cylinder configuration
  and against the reference solver's own complex amplitudes on the same polygon
  (``tests/golden/ref_cylinder_c1.npz``).  The reference discretises with linear
  Galerkin elements and an S+gamma*D combined potential, so agreement is at the
  discretisation-error level (hundredths of a dB), not bit level.
* The linear-algebra boundary (reference ``twod/solver.py:355-392``
  ``_solve_dense_gpu``) is pinned exactly on the reference's own assembled matrices
  (``tests/golden/ref_dense_system.npz``).
"""
