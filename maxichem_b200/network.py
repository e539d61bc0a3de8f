"""A VULCAN reaction list and its NASA-9 thermodynamics, read into arrays.

The reader works in three passes over the text:

1. ``scan`` turns the file into typed records: section headings (classified by the prefix table ``HEADINGS``),
   reaction lines (equation and fields), attachment lines (``Troe [...]`` or ``effi {...}``), column titles,
   commented-out reactions and free text, each with its line number.
2. ``Assembler`` walks the records as a small state machine (the section in force, and whether the thermal part has
   ended) and builds each reaction from the law table ``LAWS``: a law names the reaction kind, the coefficient names
   it reads, or a fixed coefficient set (the one "special" law), or a refusal.
3. ``VulcanNetwork`` indexes species, reads the NASA-9 files and checks the assembled network once: third bodies,
   atom balance, repeated names, photolysis species, duplicates.

The file format (the headings, the bracketed equation, the coefficient order of each law, the Troe and efficiency
lines, the photolysis absorber and branch fields, the NASA-9 layout) and the attributes of ``VulcanNetwork`` are
those of imalsky/maxichem ``maxichem/kinvulcan.py:32-357``, so a table built from a network is the same whichever
reader made it.
"""

from __future__ import annotations

import ast
import re
from dataclasses import dataclass
from pathlib import Path
from typing import Any, Iterator, NamedTuple

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

# The one law held as numbers rather than read from the file: OH + CH3 + M -> CH3OH + M (Jasper et al. 2007, as
# fitted by Visscher & Moses 2011, eqs. 13-14): two low-pressure terms, a high-pressure term and a Troe factor whose
# width follows their form ("vm11"). Format constants of the reference reader (kinvulcan.py:41-55).
SPECIAL: dict[str, dict[str, Any]] = {
    "OH+CH3+M->CH3OH+M": {
        "A0": 1.932e3, "B0": -9.88, "C0": 7544.0,
        "A1": 5.109e-11, "B1": -6.25, "C1": 1433.0,
        "Ai": 1.031e-10, "Bi": -0.018, "Ci": -16.74,
        "troe": (0.8145, 155.8, 1675.0, 4531.0),
        "width": "vm11",
    }
}  # fmt: skip


class Law(NamedTuple):
    kind: int | None  # None: the section's reactions are refused
    coefficients: tuple[str, ...]  # read from the line, in order
    fixed: bool = False  # the law's numbers come from SPECIAL, keyed by the equation


# Section name -> its rate law.
LAWS: dict[str, Law] = {
    "two": Law(KIND_TWO_BODY, ("A", "B", "C")),
    "three": Law(KIND_FALLOFF, ("A0", "B0", "C0", "Ai", "Bi", "Ci")),
    "low": Law(KIND_LOW_PRESSURE, ("A0", "B0", "C0")),
    "special": Law(KIND_SPECIAL, (), fixed=True),
    "irrev": Law(None, ()),
}

# Heading prefixes (lower case) and what they start, tried in order: the longer "3-body ... without high-pressure"
# before "3-body". "end" headings close the thermal part: photolysis follows "# photo"; condensation and the rest
# are counted and skipped; "# reverse stops" only closes.
HEADINGS: tuple[tuple[str, str], ...] = (
    ("# two-body", "two"),
    ("# 3-body reactions without high-pressure", "low"),
    ("# 3-body", "three"),
    ("# special", "special"),
    ("# irreversible", "irrev"),
    ("# reverse stops", "end"),
    ("# photo", "end:photo"),
    ("# condensation", "end:skip"),
    ("# re_end", "end:skip"),
)
_NASA_SIZES = (20, 30, 40)


def formula(name: str) -> dict[str, int]:
    """Element counts of a species name, repeats summed (CH3OH -> C 1, H 4, O 1)."""
    counts: dict[str, int] = {}
    for element, number in re.findall(r"([A-Z][a-z]?)(\d*)", name):
        counts[element] = counts.get(element, 0) + (int(number) if number else 1)
    return counts


def gibbs_rt(a: np.ndarray, T: float) -> float:
    """G/RT from one NASA-9 range a1..a7, b1, b2 (McBride et al. 2002) at T in K: H/RT - S/R."""
    lt, t2, t3, t4 = np.log(T), T * T, T**3, T**4
    h_rt = -a[0] / t2 + a[1] * lt / T + a[2] + a[3] * T / 2 + a[4] * t2 / 3 + a[5] * t3 / 4 + a[6] * t4 / 5 + a[7] / T
    s_r = -a[0] / t2 / 2 - a[1] / T + a[2] * lt + a[3] * T + a[4] * t2 / 2 + a[5] * t3 / 3 + a[6] * t4 / 4 + a[8]
    return float(h_rt - s_r)


# ---- pass 1: records ----


@dataclass
class Record:
    kind: str  # "heading", "reaction", "attach", "titles", "commented", "text", "blank"
    where: str  # file:line
    line: str
    section: str = ""  # heading: what it starts
    equation: str = ""  # reaction
    fields: tuple[str, ...] = ()  # reaction: the fields after the bracket
    problem: str = ""  # reaction: why the line is not a well-formed reaction (raised only if the line is used as one)

    def parts(self) -> tuple[str, tuple[str, ...]]:
        if self.problem:
            raise ValueError(self.problem)
        return self.equation, self.fields


def _reaction_parts(line: str, where: str) -> tuple[str, tuple[str, ...]]:
    head, bracket, tail = line.partition("[")
    inside, closing, rest = tail.partition("]")
    if not bracket or not closing:
        raise ValueError(f"{where}: a reaction line needs its equation in [ ]: {line}")
    if "->" not in inside:
        raise ValueError(f"{where}: the equation needs ->: {line}")
    return inside.strip(), tuple(rest.split())


def scan(text: str, path: str | Path) -> Iterator[Record]:
    """The file's lines as typed records."""
    for number, raw in enumerate(text.split("\n"), 1):
        line, where = raw.strip(), f"{path}:{number}"
        if not line:
            yield Record("blank", where, line)
        elif line.startswith("#"):
            low = line.lower()
            section = next((s for prefix, s in HEADINGS if low.startswith(prefix)), "")
            if section:
                yield Record("heading", where, line, section=section)
            elif low.startswith("# id"):
                yield Record("titles", where, line)
            elif "[" in low or not low.strip("# "):
                yield Record("commented", where, line)
            else:
                yield Record("text", where, line)
        elif line.startswith(("Troe", "effi")):
            yield Record("attach", where, line)
        elif "[" in line:
            try:
                equation, fields = _reaction_parts(line, where)
                yield Record("reaction", where, line, equation=equation, fields=fields)
            except ValueError as e:  # a condensation line is only counted: its form matters only where it is read
                yield Record("reaction", where, line, problem=str(e))
        else:
            yield Record("text", where, line)


# ---- pass 2: reactions ----


def _numbers(values: Any, count: int | None, what: str, rec: Record) -> list[float]:
    try:
        out = [float(v) for v in values]
    except (TypeError, ValueError):
        raise ValueError(f"{rec.where}: {what} must be numbers: {rec.line}") from None
    if count is not None and len(out) != count:
        raise ValueError(f"{rec.where}: {count} {what} expected, found {len(out)}: {rec.line}")
    if not all(np.isfinite(out)):
        raise ValueError(f"{rec.where}: finite rate coefficients expected, got {out}: {rec.line}")
    return out


def _sides(equation: str) -> tuple[list[str], list[str]]:
    left, right = equation.split("->", 1)
    return [q.strip() for q in left.split("+")], [q.strip() for q in right.split("+")]


class Assembler:
    """The records' state machine: the section in force, and whether the thermal part has ended."""

    def __init__(self, bulk: str) -> None:
        self.bulk = bulk
        self.section: str | None = None
        self.closed = False  # past an "end" heading
        self.after = ""  # after the thermal part: "photo", "skip" or "" (nothing may follow)
        self.thermal: list[dict[str, Any]] = []
        self.photo: list[dict[str, Any]] = []
        self.branches: set[tuple[str, int]] = set()
        self.skipped = 0

    def feed(self, rec: Record) -> None:
        handler = getattr(self, "on_" + rec.kind, None)
        if handler:
            handler(rec)

    def on_heading(self, rec: Record) -> None:
        kind, _, what = rec.section.partition(":")
        if kind == "end":
            self.closed = True
            if what:
                self.after = what
        elif not self.closed:
            self.section = kind

    def on_text(self, rec: Record) -> None:
        # free text is allowed above the first heading and after the thermal part; inside it, a line starting with
        # '#' that is no heading would silently keep the law of the section above, so it is refused
        if rec.line.startswith("#") and self.section is not None and not self.closed:
            known = tuple(prefix for prefix, _ in HEADINGS)
            raise ValueError(f"{rec.where}: unknown heading: {rec.line}. Known headings: {known}; free text belongs "
                             "above the first one")  # fmt: skip

    def on_attach(self, rec: Record) -> None:
        if self.closed:
            return
        if not self.thermal:
            raise ValueError(f"{rec.where}: a Troe or effi line must follow its reaction: {rec.line}")
        try:
            value = ast.literal_eval(rec.line[4:].strip())
        except (ValueError, SyntaxError):
            raise ValueError(f"{rec.where}: the list or dict of this line cannot be read: {rec.line}") from None
        target = self.thermal[-1]
        if rec.line.startswith("Troe"):
            if len(value) != 4:
                raise ValueError(f"{rec.where}: a Troe line holds 4 numbers (a, T3, T1, T2), found {len(value)}")
            target["troe"] = tuple(_numbers(value, 4, "Troe numbers", rec))
        else:
            if self.bulk not in value:
                raise ValueError(f"{rec.where}: the efficiencies name no bulk gas {self.bulk}; choose another bulk")
            target["eff"] = _numbers([value[self.bulk]], 1, "efficiencies", rec)[0]

    def on_reaction(self, rec: Record) -> None:
        if self.closed:
            if self.after == "photo":
                self.photo.append(self._branch(rec))
            elif self.after == "skip":
                self.skipped += 1
            else:
                raise ValueError(f"{rec.where}: a reaction after '# reverse stops' outside photolysis or condensation: "
                                 f"{rec.line}")  # fmt: skip
            return
        if self.section is None:
            raise ValueError(f"{rec.where}: a reaction above the first heading has no rate law: {rec.line}")
        rec.parts()
        self.thermal.append(self._thermal(rec, LAWS[self.section]))

    def _thermal(self, rec: Record, law: Law) -> dict[str, Any]:
        if law.kind is None:
            raise ValueError(f"{rec.where}: irreversible reactions have no reverse law here; drop or move "
                             f"{rec.equation}")  # fmt: skip
        left, right = _sides(rec.equation)
        r: dict[str, Any] = {"eq": rec.equation, "kind": law.kind,
                             "names": ([q for q in left if q != "M"], [q for q in right if q != "M"])}  # fmt: skip
        if law.fixed:
            numbers = SPECIAL.get(rec.equation.replace(" ", ""))
            if numbers is None:
                raise ValueError(f"{rec.where}: unknown special reaction {rec.equation}")
            r.update(numbers)
        else:
            n = len(law.coefficients)
            if len(rec.fields) < n:
                raise ValueError(f"{rec.where}: {n} rate coefficients expected, found {len(rec.fields)}: {rec.line}")
            r.update(zip(law.coefficients, _numbers(rec.fields[:n], n, "rate coefficients", rec)))
        return r

    def _branch(self, rec: Record) -> dict[str, Any]:
        rec.parts()
        if len(rec.fields) < 2:
            raise ValueError(f"{rec.where}: a photolysis line names its absorber and branch index: {rec.line}")
        left, right = _sides(rec.equation)
        absorber = rec.fields[0]
        if left != [absorber]:
            raise ValueError(f"{rec.where}: the line's reactant is not its absorber {absorber}: {rec.line}")
        try:
            branch = int(rec.fields[1])
        except ValueError:
            raise ValueError(f"{rec.where}: the branch index is not an integer: {rec.line}") from None
        if (absorber, branch) in self.branches:
            raise ValueError(f"{rec.where}: absorber {absorber} has branch {branch} twice")
        self.branches.add((absorber, branch))
        return {"eq": rec.equation, "names": (left, right), "absorber": absorber, "branch": branch}


def read_reactions(path: str | Path, bulk: str) -> tuple[list[dict[str, Any]], list[dict[str, Any]], int]:
    """Thermal reactions, photolysis branches and the number of condensation lines skipped."""
    asm = Assembler(bulk)
    for rec in scan(Path(path).read_text(), path):
        asm.feed(rec)
    return asm.thermal, asm.photo, asm.skipped


# ---- pass 3: the network and its checks ----


def check_third_body(equation: str, kind: int, where: str) -> None:
    """A three-body law has M on both sides of its equation, a two-body law on neither."""
    with_m = ["M" in side for side in _sides(equation)]
    needs = kind in THREE_BODY_KINDS
    if with_m != [needs, needs]:
        found = " and ".join(s for s, m in zip(("reactant", "product"), with_m) if m) or "no"
        rule = "on both sides (a three-body law)" if needs else "on neither side (a two-body law)"
        raise ValueError(f"{where}: M on {found} side, but this reaction's law needs M {rule}: {equation}")


def _stoichiometry(reactions: list[dict[str, Any]], ns: int) -> np.ndarray:
    s = np.zeros((ns, len(reactions)), np.float64)
    for j, r in enumerate(reactions):
        np.subtract.at(s[:, j], r.get("re", []), 1.0)
        np.add.at(s[:, j], r.get("pr", []), 1.0)
    return s


def _element_change(r: dict[str, Any]) -> dict[str, int]:
    net: dict[str, int] = {}
    for side, sign in zip(r["names"], (-1, 1)):
        for q in side:
            for e, n in formula(q.split("_")[0]).items():
                net[e] = net.get(e, 0) + sign * n
    return {e: n for e, n in net.items() if n}


def _read_nasa(path: Path) -> tuple[np.ndarray, np.ndarray]:
    """The ranges below and above NASA_SPLIT_T of one NASA-9 file: a1..a7, b1, b2 each (the entry between a7 and b1
    is unused)."""
    values = np.loadtxt(path).ravel()
    if values.size not in _NASA_SIZES:
        raise ValueError(f"{path}: {values.size} numbers; a NASA-9 file holds one of {_NASA_SIZES}")
    ranges = values[:20].reshape(2, 10)
    lo, hi = (np.delete(r, 7) for r in ranges)
    jump = abs(gibbs_rt(lo, NASA_SPLIT_T) - gibbs_rt(hi, NASA_SPLIT_T))
    if not jump <= MAX_GIBBS_JUMP:
        raise ValueError(f"{path}: G / RT jumps by {jump:.3g} at {NASA_SPLIT_T:g} K (limit {MAX_GIBBS_JUMP:g}): the "
                         "first two ranges should meet there, below and above it")  # fmt: skip
    return lo, hi


class VulcanNetwork:
    """A VULCAN reaction list with its NASA-9 data (the reference's ``VulcanNetwork``, same attributes).

    Attributes: ``species``, ``elements``, ``atoms`` [species, elements], ``lo``/``hi`` [species, 9] (a1..a7, b1, b2
    of the ranges below/above NASA_SPLIT_T), ``reac`` (thermal reaction dicts with their law), ``S`` [species,
    reactions], ``photo``/``Sp`` (photolysis branches and their stoichiometry), ``photo_missing``, ``skipped``,
    ``duplicates``.
    """

    def __init__(self, network_file: str | Path, nasa_dir: str | Path, species: list[str] | None = None,
                 bulk: str = "H2") -> None:  # fmt: skip
        thermal, photo, self.skipped = read_reactions(network_file, bulk)
        self.species = list(species) if species is not None else self._first_appearance(thermal)
        repeated = sorted({q for q in self.species if self.species.count(q) > 1})
        if repeated:
            raise ValueError(f"species names {repeated} more than once: each name is one row of the state")
        folder = Path(nasa_dir)
        missing = [q for q in self.species if not (folder / f"{q}.txt").exists()]
        if missing:
            raise FileNotFoundError(f"no NASA-9 file for {missing[0]}: {folder / (missing[0] + '.txt')}; pass the "
                                    "folder that holds one per species")  # fmt: skip
        ranges = [_read_nasa(folder / f"{q}.txt") for q in self.species]
        self.lo = np.array([r[0] for r in ranges], np.float64)
        self.hi = np.array([r[1] for r in ranges], np.float64)
        counts = [formula(q.split("_")[0]) for q in self.species]
        self.elements = sorted({e for c in counts for e in c})
        self.atoms = np.array([[c.get(e, 0) for e in self.elements] for c in counts], np.float64)
        self.reac = thermal
        self.photo = photo
        self._validate(network_file)
        self.duplicates = self._duplicates(thermal)
        self.S = _stoichiometry(thermal, len(self.species))
        self.Sp = _stoichiometry(photo, len(self.species))

    @staticmethod
    def _first_appearance(thermal: list[dict[str, Any]]) -> list[str]:
        order = list(dict.fromkeys(q for r in thermal for q in r["names"][0] + r["names"][1]))
        return order if "He" in order else order + ["He"]

    def _validate(self, network_file: str | Path) -> None:
        """The checks of the assembled network, in one pass: species indices, third bodies, atom balance of the thermal
        reactions, photolysis species and balance."""
        row = {q: i for i, q in enumerate(self.species)}
        for j, r in enumerate(self.reac):
            unknown = [q for q in r["names"][0] + r["names"][1] if q not in row]
            if unknown:
                raise ValueError(f"{network_file}: reaction {r['eq']} names {unknown}, not in the species list")
            r["re"] = [row[q] for q in r["names"][0]]
            r["pr"] = [row[q] for q in r["names"][1]]
            check_third_body(r["eq"], r["kind"], f"{network_file}: reaction {j}")
        unbalanced = [r["eq"] for r in self.reac if _element_change(r)]
        if unbalanced:
            raise ValueError(f"reactions that do not balance their atoms: {unbalanced}")
        self.photo_missing = sorted({q for r in self.photo for q in r["names"][0] + r["names"][1] if q not in row})
        for r in self.photo:
            if _element_change(r):
                raise ValueError(f"photolysis branch {r['eq']} does not balance its atoms")
            if not self.photo_missing:
                r["re"] = [row[q] for q in r["names"][0]]
                r["pr"] = [row[q] for q in r["names"][1]]

    @staticmethod
    def _duplicates(thermal: list[dict[str, Any]]) -> list[tuple[str, str]]:
        """Pairs (first, later) of reactions with the same species on the same two sides, in either direction."""
        first: dict[tuple, str] = {}
        pairs = []
        for r in thermal:
            extra = () if r["kind"] == KIND_TWO_BODY else ("M",)
            key = tuple(sorted(tuple(sorted(side)) + extra for side in r["names"]))
            if key in first:
                pairs.append((first[key], r["eq"]))
            else:
                first[key] = r["eq"]
        return pairs
