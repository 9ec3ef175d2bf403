"""CPU oracle for the fixed-charge nonbonded path (test infrastructure only; see oracle.py)."""
