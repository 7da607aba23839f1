"""CPU oracle of gample's PIC step -- test infrastructure only.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may
import this package. The product (gample_b200/) never does.
"""
