"""CPU checkers for the CUDA path (test infrastructure only; see oracle.py)."""
