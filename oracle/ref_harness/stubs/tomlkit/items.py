"""Stand-in for ``tomlkit.items``. Test infrastructure only."""


class Table(dict):
    pass


class Trivia:
    pass
