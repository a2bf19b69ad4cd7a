"""CPU oracle for the cDFT.jl ``converge!`` hot path (TEST INFRASTRUCTURE ONLY).

This package restates, in NumPy FP64, the arithmetic of the reference
(ClapeyronThermo/cDFT.jl) on the converge! path so that the CUDA library can be
checked against it.  It is imported only by ``tests/``, by
``__graft_entry__.smoke()`` and by the ``cpu_baseline`` / ``--impl reference``
legs of ``bench.py`` -- never by the product path (``cdft.jl_b200``), which
fails loudly when its CUDA library is missing.

Pinning (the reference is Julia and cannot run in this container):
  * ``anderson.aasol`` reproduces the Toth--Kelley residual histories printed in
    the docstring of src/utils/anderson.jl:116-160 (test_oracle_anderson.py);
  * ``functional`` reproduces bulk consistency, dF/drho at a uniform profile ==
    mu_res of an independent bulk PC-SAFT (``pcsaft_bulk``, written from
    Gross & Sadowski 2001/2002), the property test/test_models.jl:11-27,153-188
    and test/test_coordinate_systems.jl:1-33 assert;
  * the gamma/adsorption constants of test/test_methods.jl need Clapeyron's
    parameter database, which is absent here: those stay unpinned.
"""
