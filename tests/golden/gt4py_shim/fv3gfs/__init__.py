"""Minimal stand-in for the fv3gfs namespace package (fixture generation only)."""
