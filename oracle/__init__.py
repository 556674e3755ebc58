"""CPU oracle of the ParaTC hot path -- TEST INFRASTRUCTURE, not product code.

Only tests/, __graft_entry__.smoke() and the CPU-baseline leg of bench.py may
import this package, and only as the checker.
"""
