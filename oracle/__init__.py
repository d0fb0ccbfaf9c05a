"""CPU oracle of the optical-photon path: test infrastructure only.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
"""
