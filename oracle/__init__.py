"""CPU oracle package (test infrastructure only; see pyoracle.py)."""
