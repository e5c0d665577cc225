"""TEST INFRASTRUCTURE ONLY: the CPU oracle of the DSMC timestep.

oracle/_ref/   the reference solver built from its own sources (oracle/Makefile)
dsmc_oracle.c  a plain-C restatement of the reference's timestep routines
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs use it.
"""
