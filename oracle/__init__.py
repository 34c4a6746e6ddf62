"""CPU oracle of the flowPsi hot path -- test infrastructure (the checker).

Only the tests, the smoke check and the CPU-baseline leg of bench.py use it.
"""
from .oracle import Oracle, RefFunctions, OracleFunctions, ref_available  # noqa: F401
