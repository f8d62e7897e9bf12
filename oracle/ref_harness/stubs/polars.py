"""Permissive import stand-in for `polars` (absent offline). Test infrastructure only."""


def __getattr__(name):
    raise AttributeError(f"polars stand-in has no attribute {name!r}")
