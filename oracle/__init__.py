"""CPU oracle of the jump-cannon layout step: test infrastructure only.

Used by tests/, by __graft_entry__.smoke() as the checker and by the CPU
baseline leg of bench.py. The product library never loads it.
"""
