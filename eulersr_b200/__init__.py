"""B200-native explicit finite-volume Euler solver (EulerSR hot path)."""
__version__ = "0.1.0"
