"""Stub matplotlib for running the reference without a plotting stack."""
def use(*a, **k):
    pass
