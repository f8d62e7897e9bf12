"""Stand-in for ``tomlkit.exceptions``. Test infrastructure only."""


class ParseError(ValueError):
    pass


class TOMLKitError(Exception):
    pass
