"""PARIS grid core on one B200: host-side mirror of the reference's Fortran
subroutine interfaces over the C-ABI of libparis_b200.so (include/paris_b200.h).
"""
from . import build, capi, workloads  # noqa: F401
from . import runtime  # noqa: F401
