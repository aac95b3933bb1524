"""CPU oracle and reference harness for the LBM-DDF time step.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py (cpu_baseline and reference legs), never by the lbm_ddf_b200 package.
"""
