"""Stand-in for f90nml (only imported, never used by the fixture generator)."""


def read(path):
    raise NotImplementedError("f90nml is not available")
