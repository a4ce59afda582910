"""The tests' handle on the FP64 CPU oracle (``oracle/orc.py``) and on the
oracle's own case layer (``oracle/case.py``)."""
from oracle import case as ocase  # noqa: F401
from oracle.orc import Oracle, anisotropy, build, load, rel_l2, set_threads, threads  # noqa: F401
