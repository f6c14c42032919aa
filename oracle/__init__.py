"""TEST INFRASTRUCTURE ONLY: CPU checkers for the B200 backend (see oracle.py)."""
