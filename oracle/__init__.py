"""ORACLE — test infrastructure, not product code.

A CPU restatement of the reference's mask-cone visibility path
(oracle/cone_oracle.cpp) used only to check the CUDA library: by tests/,
__graft_entry__.smoke() and bench.py's CPU baseline. Nothing in continuum_b200
imports it.
"""
