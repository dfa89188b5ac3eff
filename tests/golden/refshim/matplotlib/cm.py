"""Stub colormap module."""
gist_rainbow = None
