"""CPU oracle of the LBM step (test infrastructure only; see oracle/oracle.py)."""
