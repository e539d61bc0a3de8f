"""A VULCAN reaction list and its NASA-9 thermodynamics, read into arrays.

The format and the refusals follow the reference reader (imalsky/maxichem ``maxichem/kinvulcan.py:32-357``):
thermal reactions under the section headings "two-body", "3-body", "3-body reactions without high-pressure",
"special" (a law held in code) and "irreversible" (refused); ``Troe [...]`` and ``effi {...}`` lines attach to the
reaction above; "# reverse stops" ends the thermal part; photolysis branches follow "# photo"; condensation lines
are counted and skipped. Species order is first appearance with He appended. The attributes match the reference's
``VulcanNetwork`` one for one, so every table built from a network is the same whichever reader made it.
"""

from __future__ import annotations

import ast
import re
from pathlib import Path
from typing import Any

import numpy as np

from .constants import (
    KIND_FALLOFF,
    KIND_LOW_PRESSURE,
    KIND_SPECIAL,
    KIND_TWO_BODY,
    MAX_GIBBS_JUMP,
    NASA_SPLIT_T,
    THREE_BODY_KINDS,
)

__all__ = ["SPECIAL", "VulcanNetwork", "formula", "gibbs_rt"]

# The one special law (kinvulcan.py:41-55): OH + CH3 + M -> CH3OH + M, Jasper et al. (2007) as fitted by Visscher &
# Moses (2011, eqs. 13-14): two k0 terms, a high-pressure term and a Troe factor without shift terms ("vm11").
SPECIAL: dict[str, dict[str, Any]] = {
    "OH+CH3+M->CH3OH+M": {
        "A0": 1.932e3,
        "B0": -9.88,
        "C0": 7544.0,
        "A1": 5.109e-11,
        "B1": -6.25,
        "C1": 1433.0,
        "Ai": 1.031e-10,
        "Bi": -0.018,
        "Ci": -16.74,
        "troe": (0.8145, 155.8, 1675.0, 4531.0),
        "width": "vm11",
    }
}

# Headings that end the thermal part (kinvulcan.py:56), and the thermal section headings in test order
# (kinvulcan.py:58-64: "# 3-body reactions without high-pressure" must be tried before "# 3-body").
_END_HEADINGS = ("# reverse stops", "# condensation", "# photo", "# re_end")
_SECTION_HEADINGS = (
    ("# two-body", "two"),
    ("# 3-body reactions without high-pressure", "low"),
    ("# 3-body", "three"),
    ("# special", "special"),
    ("# irreversible", "irrev"),
)
_KNOWN = (*_END_HEADINGS, *(h for h, _ in _SECTION_HEADINGS))
_NASA_SIZES = (20, 30, 40)


def formula(name: str) -> dict[str, int]:
    """Element counts of a species name, repeats summed (CH3OH -> C 1, H 4, O 1)."""
    counts: dict[str, int] = {}
    for element, number in re.findall(r"([A-Z][a-z]?)(\d*)", name):
        counts[element] = counts.get(element, 0) + (int(number) if number else 1)
    return counts


def gibbs_rt(a: np.ndarray, T: float) -> float:
    """G/RT from one NASA-9 range a1..a7, b1, b2 (McBride et al. 2002) at T in K."""
    lt = np.log(T)
    h = -a[0] / T**2 + a[1] * lt / T + a[2] + a[3] * T / 2 + a[4] * T**2 / 3 + a[5] * T**3 / 4 + a[6] * T**4 / 5
    s = -a[0] / T**2 / 2 - a[1] / T + a[2] * lt + a[3] * T + a[4] * T**2 / 2 + a[5] * T**3 / 3 + a[6] * T**4 / 4
    return float((h + a[7] / T) - (s + a[8]))


def _split_reaction(line: str, where: str) -> tuple[str, list[str]]:
    """``id [ A + B -> C ] fields`` -> (equation, fields)."""
    if "[" not in line or "]" not in line.split("[", 1)[1]:
        raise ValueError(f"{where}: a reaction line needs [ reaction ]: {line}")
    inside, rest = line.split("[", 1)[1].split("]", 1)
    if "->" not in inside:
        raise ValueError(f"{where}: a reaction needs ->: {line}")
    return inside.strip(), rest.split()


def _coefficients(fields: list[str], count: int, where: str, line: str) -> list[float]:
    try:
        values = [float(v) for v in fields[:count]]
    except ValueError:
        raise ValueError(f"{where}: {count} rate coefficients expected: {line}") from None
    if len(values) < count:
        raise ValueError(f"{where}: {count} rate coefficients expected, found {len(values)}: {line}")
    if not np.all(np.isfinite(values)):
        raise ValueError(f"{where}: finite rate coefficients expected, got {values}: {line}")
    return values


def check_third_body(equation: str, kind: int, where: str) -> None:
    """M on both sides for a three-body law, on neither for a two-body one (kinvulcan.py:115-127)."""
    sides = [[q.strip() for q in side.split("+")] for side in equation.split("->")]
    has_m = ["M" in side for side in sides]
    want = kind in THREE_BODY_KINDS
    if has_m != [want, want]:
        named = " and ".join(s for s, m in zip(("reactant", "product"), has_m) if m) or "no"
        need = "on both sides (a three-body law)" if want else "on neither side (a two-body law)"
        raise ValueError(f"{where}: M on {named} side, but this reaction's law needs M {need}: {equation}")


def _thermal(line: str, where: str, section: str) -> dict[str, Any]:
    equation, fields = _split_reaction(line, where)
    lhs, rhs = (side.split("+") for side in equation.split("->"))
    names = ([q.strip() for q in lhs if q.strip() != "M"], [q.strip() for q in rhs if q.strip() != "M"])
    r: dict[str, Any] = {"eq": equation, "names": names}
    if section == "two":
        r["kind"] = KIND_TWO_BODY
        r["A"], r["B"], r["C"] = _coefficients(fields, 3, where, line)
    elif section == "three":
        r["kind"] = KIND_FALLOFF
        r.update(zip(("A0", "B0", "C0", "Ai", "Bi", "Ci"), _coefficients(fields, 6, where, line)))
    elif section == "low":
        r["kind"] = KIND_LOW_PRESSURE
        r["A0"], r["B0"], r["C0"] = _coefficients(fields, 3, where, line)
    elif section == "irrev":
        raise ValueError(f"no reverse law for the irreversible reaction {equation}: the reader has none")
    else:
        key = equation.replace(" ", "")
        if key not in SPECIAL:
            raise ValueError(f"unknown special reaction {equation}")
        r["kind"] = KIND_SPECIAL
        r.update(SPECIAL[key])
    check_third_body(equation, r["kind"], where)
    return r


def _photolysis(line: str, where: str, seen: set[tuple[str, int]]) -> dict[str, Any]:
    equation, fields = _split_reaction(line, where)
    if len(fields) < 2:
        raise ValueError(f"{where}: a photolysis line needs its absorber and branch index: {line}")
    lhs, rhs = ([q.strip() for q in side.split("+")] for side in equation.split("->"))
    if lhs != [fields[0]]:
        raise ValueError(f"{where}: a photolysis line whose reactant is not its absorber {fields[0]}: {line}")
    try:
        branch = int(fields[1])
    except ValueError:
        raise ValueError(f"{where}: a photolysis branch index must be an integer: {line}") from None
    if (fields[0], branch) in seen:
        raise ValueError(f"{where}: two photolysis lines for absorber {fields[0]}, branch {branch}")
    seen.add((fields[0], branch))
    return {"eq": equation, "names": (lhs, rhs), "absorber": fields[0], "branch": branch}


def _attach(line: str, where: str, reactions: list[dict[str, Any]], bulk: str) -> None:
    """A ``Troe [...]`` or ``effi {...}`` line, for the reaction above it."""
    if not reactions:
        raise ValueError(f"{where}: this line must follow a reaction: {line}")
    try:
        value = ast.literal_eval(line[4:].strip())
    except (ValueError, SyntaxError):
        raise ValueError(f"{where}: this line's list or dict cannot be read: {line}") from None
    if line.startswith("Troe"):
        if len(value) != 4:
            raise ValueError(f"{where}: a Troe line holds 4 numbers (a, T3, T1, T2), got {len(value)}: {line}")
        troe = [float(v) for v in value]
        if not np.all(np.isfinite(troe)):
            raise ValueError(f"{where}: finite rate coefficients expected, got {troe}: {line}")
        reactions[-1]["troe"] = tuple(troe)
        return
    if bulk not in value:
        raise ValueError(f"{where}: no efficiency for the bulk gas {bulk}; pass another bulk: {line}")
    eff = float(value[bulk])
    if not np.isfinite(eff):
        raise ValueError(f"{where}: finite rate coefficients expected, got {[eff]}: {line}")
    reactions[-1]["eff"] = eff


def read_reactions(path: str | Path, bulk: str) -> tuple[list[dict[str, Any]], list[dict[str, Any]], int]:
    """Thermal reactions, photolysis branches and the number of condensation lines skipped (kinvulcan.py:191-223)."""
    reactions: list[dict[str, Any]] = []
    photo: list[dict[str, Any]] = []
    seen: set[tuple[str, int]] = set()
    section: str | None = None
    ended = False
    skipped = 0
    for number, raw in enumerate(Path(path).read_text().split("\n"), 1):
        line, where = raw.strip(), f"{path}:{number}"
        if line.startswith("#"):
            low = line.lower()
            if section is not None and not ended:
                # a comment inside the thermal part must be a known heading, column titles, a commented-out
                # reaction or empty, so an unknown heading cannot silently keep the law of the section above
                if not (low.startswith((*_KNOWN, "# id")) or "[" in low or not low.strip("# ")):
                    raise ValueError(
                        f"{where}: unknown heading: {line}. The headings are {_KNOWN}; free text goes above the first one"
                    )
            if low.startswith(_END_HEADINGS):
                ended = True
                if low.startswith("# photo"):
                    section = "photo"
                elif not low.startswith("# reverse stops"):
                    section = "skip"
            elif not ended:
                for heading, name in _SECTION_HEADINGS:
                    if low.startswith(heading):
                        section = name
                        break
            continue
        if ended:
            if "[" in line:
                if section == "photo":
                    photo.append(_photolysis(line, where, seen))
                elif section == "skip":
                    skipped += 1
                else:
                    raise ValueError(f"reaction after '# reverse stops' outside photolysis / condensation: {line}")
        elif line.startswith(("Troe", "effi")):
            _attach(line, where, reactions, bulk)
        elif "[" in line:
            if section is None:
                raise ValueError(f"{where}: a reaction above the first heading has no rate law: {line}")
            reactions.append(_thermal(line, where, section))
    return reactions, photo, skipped


def _stoichiometry(reactions: list[dict[str, Any]], ns: int) -> np.ndarray:
    s = np.zeros((ns, len(reactions)), np.float64)
    for j, r in enumerate(reactions):
        for i in r.get("re", ()):
            s[i, j] -= 1
        for i in r.get("pr", ()):
            s[i, j] += 1
    return s


class VulcanNetwork:
    """A VULCAN reaction list with its NASA-9 data (the reference's ``VulcanNetwork``, same attributes).

    Attributes: ``species``, ``elements``, ``atoms`` [species, elements], ``lo``/``hi`` [species, 9] (a1..a7, b1, b2
    of the ranges below/above NASA_SPLIT_T), ``reac`` (thermal reaction dicts with their law), ``S`` [species,
    reactions], ``photo``/``Sp`` (photolysis branches and their stoichiometry), ``photo_missing``, ``skipped``,
    ``duplicates``.
    """

    def __init__(
        self, network_file: str | Path, nasa_dir: str | Path, species: list[str] | None = None, bulk: str = "H2"
    ) -> None:
        reactions, photo, self.skipped = read_reactions(network_file, bulk)
        if species is None:
            order: list[str] = []
            for r in reactions:
                for q in r["names"][0] + r["names"][1]:
                    if q not in order:
                        order.append(q)
            if "He" not in order:
                order.append("He")
            species = order
        self.species = list(species)
        repeated = sorted({q for q in self.species if self.species.count(q) > 1})
        if repeated:
            raise ValueError(f"species names {repeated} more than once: a name is one row of the state; drop repeats")
        self.lo, self.hi = self._nasa(Path(nasa_dir))
        self.reac = reactions
        self._index(reactions, network_file)
        self.duplicates = self._find_duplicates(reactions)
        self.S = _stoichiometry(reactions, len(self.species))
        counts = [formula(q.split("_")[0]) for q in self.species]
        self.elements = sorted({e for c in counts for e in c})
        self.atoms = np.array([[c.get(e, 0) for e in self.elements] for c in counts], np.float64)
        unbalanced = [reactions[j]["eq"] for j in np.flatnonzero(np.abs(self.atoms.T @ self.S).max(0) > 0)]
        if unbalanced:
            raise ValueError(f"reactions that do not balance their atoms: {unbalanced}")
        self.photo_missing = sorted({q for r in photo for q in r["names"][0] + r["names"][1] if q not in self.species})
        for r in photo:
            balance: dict[str, int] = {}
            for side, sign in ((r["names"][0], -1), (r["names"][1], 1)):
                for q in side:
                    for e, n in formula(q.split("_")[0]).items():
                        balance[e] = balance.get(e, 0) + sign * n
            if any(balance.values()):
                raise ValueError(f"photolysis branch {r['eq']} does not balance its atoms")
        if not self.photo_missing:
            self._index(photo, network_file)
        self.photo = photo
        self.Sp = _stoichiometry(photo, len(self.species))

    def _nasa(self, folder: Path) -> tuple[np.ndarray, np.ndarray]:
        lo, hi = [], []
        for name in self.species:
            path = folder / f"{name}.txt"
            if not path.exists():
                raise FileNotFoundError(f"no NASA-9 file for {name}: {path}; pass the folder that holds it")
            a = np.loadtxt(path).flatten()
            if a.size not in _NASA_SIZES:
                raise ValueError(f"{path}: {a.size} numbers, a NASA-9 file holds {_NASA_SIZES}; check the file")
            # each range: a1..a7, an unused entry, b1, b2
            lo.append(np.concatenate([a[0:7], a[8:10]]))
            hi.append(np.concatenate([a[10:17], a[18:20]]))
            jump = abs(gibbs_rt(lo[-1], NASA_SPLIT_T) - gibbs_rt(hi[-1], NASA_SPLIT_T))
            if not jump <= MAX_GIBBS_JUMP:
                raise ValueError(
                    f"{path}: G / RT jumps by {jump:.3g} at {NASA_SPLIT_T:g} K, above {MAX_GIBBS_JUMP:g}: the two "
                    "ranges read do not meet; check that the file's first two ranges are the ones below and above it"
                )
        return np.array(lo, np.float64), np.array(hi, np.float64)

    def _index(self, reactions: list[dict[str, Any]], network_file: str | Path) -> None:
        position = {q: i for i, q in enumerate(self.species)}
        for r in reactions:
            missing = [q for q in r["names"][0] + r["names"][1] if q not in position]
            if missing:
                raise ValueError(f"{network_file}: reaction {r['eq']} names {missing}, not in the species list")
            r["re"] = [position[q] for q in r["names"][0]]
            r["pr"] = [position[q] for q in r["names"][1]]

    @staticmethod
    def _find_duplicates(reactions: list[dict[str, Any]]) -> list[tuple[str, str]]:
        seen: dict[Any, str] = {}
        found = []
        for r in reactions:
            m = ("M",) if r["kind"] != KIND_TWO_BODY else ()
            key = tuple(sorted((tuple(sorted(r["names"][0])) + m, tuple(sorted(r["names"][1])) + m)))
            if key in seen:
                found.append((seen[key], r["eq"]))
            seen.setdefault(key, r["eq"])
        return found


# Re-exported for the tables: the kinds with M and with a high-pressure rate.
KINDS = {"two": KIND_TWO_BODY, "three": KIND_FALLOFF, "low": KIND_LOW_PRESSURE, "special": KIND_SPECIAL}
