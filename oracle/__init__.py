'''CPU oracle for the Lorenz-Mie hot path -- TEST INFRASTRUCTURE ONLY.

This package restates, in plain numpy FP64, the reference algorithms of
pylorenzmie that the CUDA library replaces:

* ``mie``   -- ``Sphere.wiscombe_yang`` / ``Sphere.mie_coefficients``
  (theory/Sphere.py:91-226) and the Yang multilayer coefficients of
  lib/obsolete/sphere_coefficients.py:40-220 (input handling repaired);
* ``field`` -- ``LorenzMie.lorenzmie`` / ``scattered_field`` / ``field`` /
  ``hologram`` (theory/LorenzMie.py:113-342) and ``meshgrid``
  (lib/meshgrid.py:10-40);
* ``fit``   -- ``Optimizer.optimize`` with its default settings and
  ``Optimizer._statistics`` (analysis/Optimizer.py:102-113, 196-278), which
  call scipy's ``least_squares(method='lm')`` (MINPACK ``lmder``).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package.  It is test infrastructure that
results are compared against, never the thing measured or shipped: the product (``pylorenzmie_b200``) never imports it.

Pinning: ``tests/golden/make_golden.py`` imports the reference itself and
writes the fixtures in ``tests/golden/``; ``tests/test_oracle_golden.py``
checks this oracle against them.  The layered-sphere restatement is pinned
only through its one-layer case and the equal-index reduction to the
homogeneous sphere (the reference's multilayer entry point cannot run on
list input), so multilayer values beyond that are "parity unpinned".
'''
