"""Permissive import stand-in for `pint` (absent offline). Test infrastructure only."""


def __getattr__(name):
    raise AttributeError(f"pint stand-in has no attribute {name!r}")
