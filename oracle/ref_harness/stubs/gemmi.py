"""Minimal P1-only ``gemmi`` stand-in for importing the reference offline.

Test infrastructure only. Covers ``read_small_structure`` for CIFs whose
only symmetry operation is the identity, and ``Op`` for that identity.
"""

import re
from types import SimpleNamespace

import numpy as np


class Op:
    def __init__(self, triplet="x,y,z"):
        self.triplet = triplet.replace(" ", "").lower()

    def __eq__(self, other):
        return isinstance(other, Op) and other.triplet == self.triplet

    def __hash__(self):
        return hash(self.triplet)

    def apply_to_xyz(self, xyz):
        if self.triplet != "x,y,z":
            raise NotImplementedError("P1 gemmi stand-in applies only the identity")
        return list(xyz)


def _num(text):
    return float(re.sub(r"\(.*?\)", "", text))


def read_small_structure(path):
    lines = open(path).read().splitlines()
    vals = {}
    for line in lines:
        parts = line.split()
        if len(parts) >= 2 and parts[0].startswith("_cell_"):
            vals[parts[0]] = _num(parts[1])
    a, b, c = vals["_cell_length_a"], vals["_cell_length_b"], vals["_cell_length_c"]
    al, be, ga = (vals["_cell_angle_alpha"], vals["_cell_angle_beta"], vals["_cell_angle_gamma"])
    ca, cb, cg = (np.cos(np.radians(x)) for x in (al, be, ga))
    volume = a * b * c * np.sqrt(1 - ca * ca - cb * cb - cg * cg + 2 * ca * cb * cg)
    sites, symops = [], []
    i = 0
    while i < len(lines):
        line = lines[i].strip()
        if line == "loop_":
            headers = []
            i += 1
            while i < len(lines) and lines[i].strip().startswith("_"):
                headers.append(lines[i].strip().split()[0])
                i += 1
            rows = []
            while i < len(lines) and lines[i].strip() and not lines[i].strip().startswith(("_", "loop_")):
                rows.append(lines[i].strip())
                i += 1
            if any("symop_operation_xyz" in h or "equiv_pos_as_xyz" in h for h in headers):
                col = [k for k, h in enumerate(headers) if "xyz" in h][0]
                for row in rows:
                    tok = re.findall(r"'[^']*'|\S+", row)
                    symops.append(tok[col].strip("'"))
            elif "_atom_site_fract_x" in headers:
                h = {name: k for k, name in enumerate(headers)}
                for row in rows:
                    tok = row.split()
                    sym = tok[h["_atom_site_type_symbol"]] if "_atom_site_type_symbol" in h else tok[h["_atom_site_label"]]
                    sym = re.match(r"[A-Za-z]+", sym).group(0)
                    sym = sym[0].upper() + sym[1:].lower()
                    occ = _num(tok[h["_atom_site_occupancy"]]) if "_atom_site_occupancy" in h else 1.0
                    fr = SimpleNamespace(
                        x=_num(tok[h["_atom_site_fract_x"]]),
                        y=_num(tok[h["_atom_site_fract_y"]]),
                        z=_num(tok[h["_atom_site_fract_z"]]),
                    )
                    sites.append(SimpleNamespace(element=SimpleNamespace(name=sym), fract=fr, occ=occ))
            continue
        i += 1
    if not symops:
        symops = ["x,y,z"]
    if any(op.replace(" ", "").lower() != "x,y,z" for op in symops):
        raise NotImplementedError(f"{path}: P1 gemmi stand-in cannot expand non-P1 symmetry")
    cell = SimpleNamespace(parameters=(a, b, c, al, be, ga), volume=volume)
    return SimpleNamespace(cell=cell, sites=sites, symops=symops, spacegroup=None)
