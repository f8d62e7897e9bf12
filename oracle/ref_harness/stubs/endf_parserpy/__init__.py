"""Import stand-in for ``endf_parserpy`` (absent offline). Test infrastructure only."""

__version__ = "0.19.0"


def __getattr__(name):
    raise AttributeError(f"endf_parserpy stand-in has no attribute {name!r}")


class EndfFile:
    def __init__(self, *args, **kwargs):
        raise RuntimeError("endf_parserpy stand-in cannot read ENDF files")


class EndfParserPy(EndfFile):
    pass
