"""Permissive import stand-in for `easygdf` (absent offline). Test infrastructure only."""


def __getattr__(name):
    raise AttributeError(f"easygdf stand-in has no attribute {name!r}")
