"""FP64 CPU oracle of the coupled lattice-Boltzmann / phase-field step.

TEST INFRASTRUCTURE ONLY.  Only the tests, the smoke check and the benchmark's
CPU legs import this package; the product (the CUDA library and its Python
host side) never loads, calls or links anything here.

* ``oracle.case``: the oracle's own reading of a BoltzTechs XML case
  (parameters, initial fields, seeded case generators), written separately
  from the product's case layer so that a fault there cannot hide in both.
* ``oracle.orc``: ctypes wrapper of ``oracle/_build/liboracle.so`` (the FP64
  OpenMP restatement of the method, ``oracle/mk_oracle.cpp``).
"""
