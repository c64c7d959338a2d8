"""dnlPython - DynELA's Python model API on the B200 engine (placeholder while the API mirror is written)."""
