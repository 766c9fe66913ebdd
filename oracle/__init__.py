"""CPU oracle of the spectral-viscosity incompressible Euler path.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py as the checker.  The product never uses it.
"""
