"""CPU oracle of the weak-weak per-turn loop -- TEST INFRASTRUCTURE ONLY.

Importable only by tests/, __graft_entry__.smoke() and the cpu_baseline leg
of bench.py, always as the checker.  The product (mbtrack_b200, libmbt)
never imports, links or calls anything here.
"""
