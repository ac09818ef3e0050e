"""Parity oracle (test infrastructure only; see orc.py)."""
