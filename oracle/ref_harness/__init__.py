"""Import the reference implementation (PyRITE v0.36.2) in a container without its data.

TEST INFRASTRUCTURE ONLY. Nothing in ``pyrite_b200`` imports this package.
It is used by ``tests/golden/make_golden.py`` to run the reference's own
CPU code and record golden vectors, and by the CPU tests that re-check the
oracle against the reference when the reference tree is present.

What it does, following the reference's own configuration seams:

* puts the reference's ``src`` on ``sys.path`` and the stand-ins under
  ``stubs/`` first (``gemmi`` P1-only reader, placeholder ``xraydb``, empty
  ``tomlkit``/``h5py``/``pint``/``polars``/``easygdf``/``endf_parserpy``);
* pins ``PYRITE_MC_BACKEND=cpu`` and ``PYRITE_MATH=reproducible`` as the
  reference's own test suite does (``tests/conftest.py:22-50``);
* points ``PYRITE_CATALOG`` (``pyrite/console/config.py:53,276``) at a copy of
  the bundled catalog with the four non-P1 crystals removed, since the
  ``gemmi`` stand-in cannot expand space-group symmetry.

The reference's numbers produced through this harness are exact for the
arithmetic of the hot path (transport with screened-Rutherford elastic and
spliced stopping; the CXR line chain, bin means, Bethe-Heitler) and
non-physical for anything read from the placeholder ``xraydb``.
"""

from __future__ import annotations

import os
import shutil
import sys
import tempfile
from pathlib import Path

HERE = Path(__file__).resolve().parent
_NON_P1 = ("gep", "ges", "gese", "gese2")


def _root(root) -> Path | None:
    """The reference tree: the ``root`` argument, else $PYRITE_REFERENCE_ROOT."""
    if root is None:
        env = os.environ.get("PYRITE_REFERENCE_ROOT")
        return Path(env) if env else None
    return Path(root)


def reference_available(root=None) -> bool:
    r = _root(root)
    return r is not None and (r / "src" / "pyrite" / "__init__.py").is_file()


def _trimmed_catalog(root: Path) -> Path:
    src = root / "src" / "pyrite" / "data" / "catalog"
    dst = Path(tempfile.gettempdir()) / "pyrite_b200_ref_catalog_v2"
    if not (dst / "catalog.toml").is_file():
        if dst.exists():
            shutil.rmtree(dst)
        shutil.copytree(src, dst)
        for name in _NON_P1:
            for sub in ("crystals", "materials"):
                for path in (dst / sub).glob(f"{name}.toml"):
                    path.unlink()
    return dst


def import_reference(root=None):
    """Return the reference ``pyrite`` package, imported through the stand-ins.
    ``root`` is the reference tree (or set $PYRITE_REFERENCE_ROOT)."""
    if not reference_available(root):
        raise RuntimeError(f"reference tree not found (root={root!r}, PYRITE_REFERENCE_ROOT="
                           f"{os.environ.get('PYRITE_REFERENCE_ROOT')!r})")
    root = _root(root)
    os.environ["PYRITE_MC_BACKEND"] = "cpu"
    os.environ["PYRITE_MATH"] = "reproducible"
    os.environ.setdefault("NUMBA_NUM_THREADS", "1")
    os.environ["PYRITE_CATALOG"] = str(_trimmed_catalog(root))
    stubs = str(HERE / "stubs")
    if stubs not in sys.path:
        sys.path.insert(0, stubs)
    src = str(root / "src")
    if src not in sys.path:
        sys.path.insert(1, src)
    import pyrite  # noqa: PLC0415

    return pyrite
