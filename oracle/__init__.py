"""CPU oracle for the batched multistatic FDTD path — TEST INFRASTRUCTURE ONLY.

Everything in this package is a plain NumPy restatement of the reference
project's algorithms (``shahzaibshazoo/ceep-v1``), written to check the CUDA
path.  Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import it; the product package ``ceep_b200`` never does, and
its GPU path fails loudly instead of falling back to anything here.

Parity pins:
  * ``fdtd2d`` (region map, CPML, source, probes) is pinned against fixtures
    produced by the reference's own ``BatchedFDTD2D.run()`` (FP64 and FP32,
    see ``tests/golden/make_golden.py``) and against ``ceep_results.json``.
  * ``fdtd3d`` is pinned against the reference's ``BatchedFDTD3D.run()``.
  * ``spectral`` (DFT, S layout, DAS) is pinned against the reference's
    ``DFTMonitor``, ``DelayAndSumBeamformer`` and ``das_imaging``.
  * The Debye/Lorentz ADE on the batched path has no reference
    implementation; it is pinned against a composition of the reference's
    ``DispersiveManager`` with its batched step (fixture ``ade2d_*``).
"""
