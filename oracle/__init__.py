"""CPU oracle (test infrastructure): see ``oracle/sgh_oracle.py``."""
