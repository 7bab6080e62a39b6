"""CPU oracle for thick_ptycho_b200 -- TEST INFRASTRUCTURE ONLY.

This package restates, in complex128 NumPy/SciPy, the algorithms of the
reference thick_ptycho paraxial (PWE) and multislice (MS) forward paths.
It is the checker of the CUDA path: only ``tests/``, ``__graft_entry__.smoke()``
and the ``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import
it.  The product package never imports it and never falls back to it.

Parity pin: the restatement is checked against golden vectors produced by the
unmodified reference (``tests/golden/make_golden.py``) in
``tests/test_oracle_golden.py``.
"""
