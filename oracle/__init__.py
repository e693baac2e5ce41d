"""CPU oracle for the FLIP liquid step of 水理ラボ (suiri-lab).

TEST INFRASTRUCTURE ONLY. Nothing in the product path imports this package: only
``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / reference arm
may use it, and only as the checker (or the timed CPU baseline), never as the thing
measured or shipped.

It is a NumPy restatement of the reference's CPU solver
(``blender_addon/suiri_lab/solver.py``), which itself is a port of the web version's WGSL
kernels (``src/js/30-wgsl-sim.js``, ``src/js/31-wgsl-sim2.js``, ``src/js/64-ripple.js``).
Every function cites the reference lines it follows. The restatement is pinned against
fixtures produced by running the reference ``solver.py`` itself
(``tests/golden/make_golden.py`` → ``tests/golden/*.npz``).

Modules:
  sdf     analytic obstacle signed distances (WGSL shape library) and the half-cell lattice
  flip    one tank: binning, P2G, forces, divergence, FP32 red-black SOR, projection, G2P,
          sub-grid drops, whitewater spawn and advance, the frame step
  ripple  top-view height map, ripple absorption mask, capillary-gravity ripple layer
  hashrng the integer hash RNG the GPU path uses (for exact spawn-decision parity)
"""
