"""Import-only stand-in used by make_golden.py (no window is ever opened)."""


def __getattr__(name):
    raise AttributeError(f"moderngl stand-in has no {name}")
