"""Permissive import stand-in for `h5py` (absent offline). Test infrastructure only."""


def __getattr__(name):
    raise AttributeError(f"h5py stand-in has no attribute {name!r}")
