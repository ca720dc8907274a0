"""Timing level switch (the reference's core/timing.py LEVEL)."""
LEVEL = 0
