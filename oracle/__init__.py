"""CPU checkers for the PDHG engine -- test infrastructure only (see oracle.py)."""
