"""Oracle for r2splat_b200 -- TEST INFRASTRUCTURE ONLY.

CPU restatements of the reference algorithms (MedAPT-group/R2Splat) used to
check the CUDA path: only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / reference legs of ``bench.py`` may import anything here, and
only as the checker. The product package never imports this directory.

* ``dense``  -- float64 PyTorch restatement of the reference's dense test
  oracle (``tests/_reference.py:13-116``): every sample evaluated, optional
  tile mask, autograd for VJPs.
* ``tiles``  -- numpy restatement of the tile intersection logic
  (``IsectTilesKernel.cu:30-273``, ``IsectTiles3DKernel.cu:36-276``) with a
  stable sort, for bit-exact comparison of counts / keys / ids / offsets.
* ``losses`` -- numpy TV / L1 restatements (``VolumeLossFwd.cu:39-82``,
  ``VolumeLossBwd.cu:46-115``, ``Loss.cpp:115-188``).
* ``build_ref`` / ``ref_ops`` -- build and load the reference's own CUDA
  sources (compiled unmodified into ``oracle/_ref/``) to compare against the
  reference implementation itself on the GPU.

Pinning: ``tests/test_oracle_golden.py`` checks these restatements against the
reference's golden vectors and known answers (``tests/golden/``, generated by
``tests/golden/make_golden.py`` from the reference checkout).
"""
