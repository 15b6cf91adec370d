"""B200-native multi-domain TDBEM time march (drop-in for the reference's
DynaGMRESSolverMultiDomainCCSR)."""
from . import cases  # noqa: F401
