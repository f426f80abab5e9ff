"""Test infrastructure: the CPU checkers of the path tracer (see checkers.py)."""
