"""Readers for EU3D's input files: mechanism, thermo, ctrl/grid/init.

The file formats are the reference's and are read with the reference's own
rules, so a case set up for EU3D runs unchanged here:

* mechanism (``input/H2_JA919.txt``): ``Reaction::ReactionRead``,
  src/Reaction.cpp:150-283 -- line 3 holds ``NS NR TB`` (tab separated);
  from line 9, 2*NR tab-separated stoichiometry rows (forward, backward per
  reaction); from line 49 (= 8 + 2*NR + 2 + 1), NR whitespace-token rows
  ``index A b Ea``; after ``NR + 3`` more lines, TB third-body rows
  ``reaction_index eff_1 .. eff_NS`` read as integers.
* thermo (``input/thermo.dat``): src/Reaction.cpp:286-320 -- from line 16,
  per species 19 whitespace tokens (9 low-range, 9 high-range NASA-9
  coefficients a1..a7,b1,b2, then the molar mass), species blocks 6 lines
  apart.
* ctrl/grid/init key/value files: ``FileReader::readFile``,
  src/FileReader.cpp:53-84 -- first two whitespace tokens of each line,
  skipped when either starts with ``#``.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Dict, List

import numpy as np

R_UNIVERSAL = 8.31434  # `R` in include/Reaction.hpp:269 and include/Flowfield.hpp:54


@dataclasses.dataclass
class Mechanism:
    """Mechanism and thermo tables in the reference's layouts.

    stoi_f, stoi_b, react_tb: (NS, NR) like ``Array<double,2> Stoi_F(NS, NR)``.
    c0, c1: (9, NS) like ``Coeff0(9, NS)``; rows a1..a7, b1, b2.
    """

    NS: int
    NR: int
    TB: int
    stoi_f: np.ndarray
    stoi_b: np.ndarray
    react_tb: np.ndarray
    af: np.ndarray
    bf: np.ndarray
    eaf: np.ndarray
    c0: np.ndarray
    c1: np.ndarray
    mw: np.ndarray
    species: List[str]

    @property
    def ri(self) -> np.ndarray:
        """Species gas constants R/Mw in kJ/(kg K), src/Reaction.cpp:352-353."""
        return R_UNIVERSAL / self.mw

    def to_json(self) -> dict:
        d = dataclasses.asdict(self)
        for k, v in d.items():
            if isinstance(v, np.ndarray):
                d[k] = v.tolist()
        return d

    @staticmethod
    def from_json(d: dict) -> "Mechanism":
        kw = dict(d)
        for k in ("stoi_f", "stoi_b", "react_tb", "af", "bf", "eaf", "c0", "c1", "mw"):
            kw[k] = np.asarray(d[k], dtype=np.float64)
        return Mechanism(**kw)


def _stoi_token(item: str) -> int:
    # std::stoi: optional leading whitespace, sign, then digits
    s = item.lstrip()
    n = 0
    while n < len(s) and (s[n].isdigit() or (n == 0 and s[n] in "+-")):
        n += 1
    if n == 0 or s[:n] in "+-":
        raise ValueError(f"stoi: no conversion for {item!r}")
    return int(s[:n])


def _istream_int(tok: str) -> int:
    # `stringstream >> int` on a token such as "6." reads the leading integer
    return _stoi_token(tok)


def read_mechanism(mech_path: str, thermo_path: str) -> Mechanism:
    """Read a mechanism file and a thermo file exactly as ReactionRead does."""
    with open(mech_path, "r", newline="", encoding="latin-1") as fh:
        lines = fh.read().split("\n")
    head = [_stoi_token(t) for t in lines[2].split("\t") if t != ""]
    NS, NR, TB = head[0], head[1], head[2]
    species = lines[4].split()[:NS]
    stoi_f = np.zeros((NS, NR))
    stoi_b = np.zeros((NS, NR))
    line = 8
    for j in range(NR):
        for arr, row in ((stoi_f, lines[line + 2 * j]), (stoi_b, lines[line + 2 * j + 1])):
            items = row.split("\t")
            if items and items[-1] == "":
                items = items[:-1]
            for i, it in enumerate(items):
                arr[i, j] = _stoi_token(it)
    line = line + 2 * NR + 2
    toks = " ".join(lines[line:]).split()
    af = np.zeros(NR)
    bf = np.zeros(NR)
    eaf = np.zeros(NR)
    t = 0
    for j in range(NR):
        b = [float(x) for x in toks[t:t + 4]]
        t += 4
        af[j], bf[j], eaf[j] = b[1], b[2], b[3]
    line = line + NR + 3
    toks = " ".join(lines[line:]).split()
    react_tb = np.zeros((NS, NR))
    t = 0
    for _ in range(TB):
        a = [_istream_int(x) for x in toks[t:t + NS + 1]]
        t += NS + 1
        for k in range(NS):
            react_tb[k, a[0] - 1] = a[k + 1]

    with open(thermo_path, "r", newline="", encoding="latin-1") as fh:
        tl = fh.read().split("\n")
    c0 = np.zeros((9, NS))
    c1 = np.zeros((9, NS))
    mw = np.zeros(NS)
    line = 15
    for j in range(NS):
        toks = " ".join(tl[line:]).split()
        aa = [float(x) for x in toks[:19]]
        c0[:, j] = aa[0:9]
        c1[:, j] = aa[9:18]
        mw[j] = aa[18]
        line += 6
    return Mechanism(NS, NR, TB, stoi_f, stoi_b, react_tb, af, bf, eaf, c0, c1, mw, species)


def read_keyvalue(path: str) -> Dict[str, str]:
    """FileReader::readFile, src/FileReader.cpp:53-84 (values kept as text)."""
    out: Dict[str, str] = {}
    with open(path, "r", encoding="latin-1") as fh:
        for line in fh:
            parts = line.split()
            if len(parts) < 2:
                continue
            k, v = parts[0], parts[1]
            if k.startswith("#") or v.startswith("#"):
                continue
            out[k] = v
    return out


@dataclasses.dataclass
class Grid:
    """Per-rank node coordinates as Mesh::Initial/Boundary build them
    (src/Mesh.cpp:75-130), for a single rank unless a block is given."""

    ni: int
    nj: int
    nk: int
    bc: int
    xnode: np.ndarray
    ynode: np.ndarray
    znode: np.ndarray


def _axis(total: int, a: float, b: float, blocks: int, rank: int, bc: int, fixed_ghosts: bool):
    d = (b - a) / (total - 1)
    n = (total - 1) // blocks + 1
    node = np.zeros(n + 2 * bc)
    for i in range(bc, n + bc):
        node[i] = a + (rank * (n - 1) + i - bc) * d
    for i in range(bc):
        if fixed_ghosts:
            # uniform extrapolation of the end spacing
            node[i] = node[bc] - (bc - i) * (node[bc + 1] - node[bc] if n > 1 else d)
            node[n + bc + i] = node[n + bc - 1] + (i + 1) * (node[n + bc - 1] - node[n + bc - 2] if n > 1 else d)
        else:
            # Mesh::Boundary, src/Mesh.cpp:110-130.  For n <= bc the lower ghost
            # reads an upper ghost node that is not yet set (zero), which makes
            # node[1] - node[0] negative.
            node[i] = 2 * node[bc] - node[2 * bc - i]
            node[n + bc + i] = 2 * node[n + bc - 1] - node[n + bc - 1 - i - 1]
    return n, node


def make_grid(total_ni: int, xa: float, xb: float, total_nj: int, ya: float, yb: float, total_nk: int,
              za: float, zb: float, bc: int = 2, blocks=(1, 1, 1), rank=(0, 0, 0),
              fixed_ghosts: bool = False) -> Grid:
    """Node coordinates of one rank.  fixed_ghosts=False reproduces the
    reference's ghost-node construction exactly; True extrapolates the ghost
    nodes with the grid spacing (the correction used by the fixed policy)."""
    ni, xn = _axis(total_ni, xa, xb, blocks[0], rank[0], bc, fixed_ghosts)
    nj, yn = _axis(total_nj, ya, yb, blocks[1], rank[1], bc, fixed_ghosts)
    nk, zn = _axis(total_nk, za, zb, blocks[2], rank[2], bc, fixed_ghosts)
    return Grid(ni, nj, nk, bc, xn, yn, zn)


def read_grid(path: str, blocks=(1, 1, 1), rank=(0, 0, 0), fixed_ghosts: bool = False) -> Grid:
    kv = read_keyvalue(path)
    g = lambda k: float(kv[k])
    return make_grid(int(g("total_ni")), g("xa"), g("xb"), int(g("total_nj")), g("ya"), g("yb"),
                     int(g("total_nk")), g("za"), g("zb"), int(g("bc")), blocks, rank, fixed_ghosts)


def stoichiometric_h2_air(mech: Mechanism) -> np.ndarray:
    """Mass fractions of H2:O2:N2 = 2:1:3.76 (molar) in the mechanism's order."""
    x = np.zeros(mech.NS)
    x[mech.species.index("H2")] = 2.0
    x[mech.species.index("O2")] = 1.0
    x[mech.species.index("N2")] = 3.76
    y = x * mech.mw
    return y / y.sum()


def molar_to_mass(mech: Mechanism, moles: Dict[str, float]) -> np.ndarray:
    x = np.zeros(mech.NS)
    for k, v in moles.items():
        x[mech.species.index(k)] = v
    y = x * mech.mw
    return y / y.sum()


def assert_finite(a: np.ndarray, what: str) -> None:
    if not np.all(np.isfinite(a)):
        raise FloatingPointError(f"{what} holds non-finite values")


__all__ = ["Mechanism", "read_mechanism", "read_keyvalue", "Grid", "make_grid", "read_grid",
           "stoichiometric_h2_air", "molar_to_mass", "R_UNIVERSAL", "assert_finite", "math"]


def load_h2_ja919() -> Mechanism:
    """The H2_JA919 mechanism with the thermo.dat tables, as parsed from the
    reference's input files into eu3d_b200/data/h2_ja919.json."""
    import json
    import os
    p = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "h2_ja919.json")
    with open(p) as fh:
        return Mechanism.from_json(json.load(fh))
