"""Import stand-in for ``tomlkit`` (absent offline). Test infrastructure only.

Reading goes through the standard library's ``tomllib``; writing is refused.
"""

import tomllib


def parse(text):
    return tomllib.loads(text)


loads = parse


def dumps(*args, **kwargs):
    raise RuntimeError("tomlkit stand-in cannot write TOML")


def document():
    return {}


def table():
    return {}


class TOMLDocument(dict):
    pass


def __getattr__(name):
    raise AttributeError(f"tomlkit stand-in has no attribute {name!r}")
