"""Seeded synthetic networks and cell inputs standing in for the VULCAN networks and GCM states.

The real VULCAN-JAX networks (NCHO_photo, 69 species; SNCHO_photo_2025, 91 species) are not available here, so each
workload runs on a seeded synthetic network of the same size, written in VULCAN's own text format with a NASA-9 file
per species and read back through the reader like any other network:

* ``cho41``: 41 C-H-O species (He last), 207 reversible reactions, 36 photolysis branches;
* ``chno69``: 69 C-H-N-O species (N via NH3/N2/HCN families), 390 reactions, 48 branches;
* ``sncho91``: 91 S-N-C-H-O species (H2S/SO2/S2/OCS families), 532 reactions, 61 branches.

Reactions balance their atoms, have at most 3 species per side, and split 60 % bimolecular, 25 % three-body
(falloff, some with Troe lines and bulk efficiencies, some low-pressure only, plus the one special law) and 15 %
unimolecular. Arrhenius A is log-uniform in 1e-16..1e-9 cm^3 s^-1 (three-body k0 divided by the number density at
1e6 dyn cm^-2 and 1000 K so it passes the collision limit there), n uniform in -2..2, Ea/R uniform in 0..3e4 K;
unimolecular A is log-uniform in 1e-4..1e4 s^-1. NASA-9 fits are two ranges continuous in H and S at 1000 K, built
so the network's equilibrium at 1500 K and 1 bar holds H2 dominant, H2O/CO/CH4 (and N2/NH3, H2S) as the heavy-element
carriers and every other species as a trace, as in hot hydrogen atmospheres.
"""

from __future__ import annotations

import hashlib
import os
from dataclasses import dataclass
from pathlib import Path
from typing import Any

import numpy as np

from .constants import KB
from .network import VulcanNetwork, formula

__all__ = ["NETWORKS", "Workload", "network", "network_files", "solar_state", "workload"]

_ROOT = Path(__file__).resolve().parent.parent

_CHO = (
    "H H2 O OH H2O O2 HO2 H2O2 C CH CH2 CH3 CH4 C2 C2H C2H2 C2H3 C2H4 C2H5 C2H6 CO CO2 HCO H2CO CH2OH CH3O "
    "CH3OH CH3CO CH2CO HCCO CH3CHO C2H5OH C3H3 C3H4 C4H2 C4H3 C6H6 HCOOH CH2CHO C3H2"
).split()
_N = (
    "N N2 NH NH2 NH3 N2H N2H2 N2H3 N2H4 HCN HNC CN NO NO2 N2O HNO HNO2 HNCO NCO CH3NH2 CH2NH C2N2 H2CN "
    "NH2OH NO3 HONO CH3CN C3N"
).split()
_S = "S S2 S3 S4 SH H2S SO SO2 SO3 OCS CS CS2 HS2 H2S2 HSO NS HCS CH3SH S2O H2SO4 CH3S C2S".split()


@dataclass(frozen=True)
class Spec:
    """A synthetic network's size and seed."""

    species: tuple[str, ...]  # without He, which the reader appends last
    reactions: int
    branches: int
    seed: int


NETWORKS: dict[str, Spec] = {
    "cho41": Spec(tuple(_CHO), 207, 36, 41),
    "chno69": Spec(tuple(_CHO + _N), 390, 48, 69),
    "sncho91": Spec(tuple(_CHO + _N + _S), 532, 61, 91),
}

_T_REF, _P_REF = 1500.0, 1e6  # K, dyn cm^-2: where the equilibrium targets hold
_ND_COLLISION = 1e6 / (KB * 1000.0)  # cm^-3: three-body k0 are scaled by this
# Equilibrium mole fractions at (_T_REF, _P_REF) of the carriers; their G/RT is 0 and they fix the element potentials
_CARRIERS = {"H2": 0.84, "He": 0.14, "H2O": 4e-4, "CO": 2.5e-4, "N2": 3e-5, "H2S": 3e-5}


def _vector(name: str, elements: list[str]) -> tuple[int, ...]:
    c = formula(name.split("_")[0])
    return tuple(c.get(e, 0) for e in elements)


def _thermo(species: list[str], elements: list[str], rng: np.random.Generator) -> dict[str, list[list[float]]]:
    """NASA-9 ranges (low, high; each a1..a7, b1, b2) from equilibrium targets at _T_REF."""
    vec = {q: np.array(_vector(q, elements), float) for q in species}
    e = {x: i for i, x in enumerate(elements)}
    lam = np.zeros(len(elements))
    lam[e["H"]] = np.log(_CARRIERS["H2"]) / 2
    lam[e["He"]] = np.log(_CARRIERS["He"])
    lam[e["O"]] = np.log(_CARRIERS["H2O"]) - 2 * lam[e["H"]]
    lam[e["C"]] = np.log(_CARRIERS["CO"]) - lam[e["O"]]
    if "N" in e:
        lam[e["N"]] = np.log(_CARRIERS["N2"]) / 2
    if "S" in e:
        lam[e["S"]] = np.log(_CARRIERS["H2S"]) - 2 * lam[e["H"]]
    out = {}
    for q in species:
        atoms = int(vec[q].sum())
        if q in _CARRIERS:
            lx = np.log(_CARRIERS[q])
        elif q == "CH4":
            lx = np.log(2e-6)
        elif q == "NH3":
            lx = np.log(3e-7)
        else:
            lx = -np.log(10.0) * (rng.uniform(5.0, 13.0) + 1.1 * max(0, atoms - 3))
        g = -lx + float(vec[q] @ lam)  # G/RT at _T_REF
        s_ref = 15.0 + 3.5 * atoms + rng.uniform(-2.0, 2.0)  # S/R at _T_REF
        h_ref = _T_REF * (g + s_ref)  # H/R at _T_REF, K
        cp = 2.5 if atoms == 1 else (3.5 if atoms == 2 else min(15.0, 4.0 + 1.0 * (atoms - 2) + rng.uniform(0, 0.5)))
        # high range: Cp/R = cph + c4h T; low range: Cp/R = cpl + c4l T + c5l T^2, Cp continuous at 1000 K
        c4l = 1e-4 * atoms * rng.uniform(0.5, 1.5) if atoms > 1 else 0.0
        c5l = -c4l / 5000.0
        cph = cp + 1000.0 * c4l + 1e6 * c5l
        c4h = 1e-5 * atoms * rng.uniform(0.0, 1.0) if atoms > 1 else 0.0
        cph -= 1000.0 * c4h
        b1h = h_ref - (cph * _T_REF + c4h * _T_REF**2 / 2)
        b2h = s_ref - (cph * np.log(_T_REF) + c4h * _T_REF)
        t = 1000.0
        h_t = cph * t + c4h * t**2 / 2 + b1h
        s_t = cph * np.log(t) + c4h * t + b2h
        b1l = h_t - (cp * t + c4l * t**2 / 2 + c5l * t**3 / 3)
        b2l = s_t - (cp * np.log(t) + c4l * t + c5l * t**2 / 2)
        low = [0.0, 0.0, cp, c4l, c5l, 0.0, 0.0, b1l, b2l]
        high = [0.0, 0.0, cph, c4h, 0.0, 0.0, 0.0, b1h, b2h]
        out[q] = [low, high]
    return out


def _arrhenius(rng: np.random.Generator, lo: float, hi: float, n: float = 2.0, ea: float = 3e4) -> str:
    a = 10.0 ** rng.uniform(np.log10(lo), np.log10(hi))
    return f"{a:.4E}  {rng.uniform(-n, n):.3f}  {rng.uniform(0.0, ea):.1f}"


def _build_text(spec: Spec, rng: np.random.Generator) -> tuple[str, list[str]]:
    """The network file's text and the species it names (He last)."""
    species = list(spec.species)
    elements = sorted({x for q in species + ["He"] for x in formula(q)})
    vec = {q: _vector(q, elements) for q in species}
    molecules = [q for q in species if sum(vec[q]) >= 2]
    pairs: dict[tuple[int, ...], list[tuple[str, str]]] = {}
    for i, a in enumerate(species):
        for b in species[i:]:
            pairs.setdefault(tuple(x + y for x, y in zip(vec[a], vec[b])), []).append((a, b))

    def split(q: str) -> list[tuple[str, str]]:
        return [p for p in pairs.get(vec[q], []) if q not in p]

    seen: set[Any] = set()

    def key(lhs: tuple[str, ...], rhs: tuple[str, ...]) -> Any:
        return tuple(sorted((tuple(sorted(lhs)), tuple(sorted(rhs)))))

    two, three, low, uni = [], [], [], []
    n3 = round(0.25 * spec.reactions)
    nu = round(0.15 * spec.reactions)
    n2 = spec.reactions - n3 - nu
    special = all(q in species for q in ("OH", "CH3", "CH3OH"))
    if special:
        seen.add(key(("OH", "CH3"), ("CH3OH",)))
        n3 -= 1

    def add_three(q: str) -> bool:
        options = [p for p in split(q) if key(p, (q,)) not in seen]
        if not options:
            return False
        a, b = options[rng.integers(len(options))]
        seen.add(key((a, b), (q,)))
        (low if rng.random() < 0.25 else three).append((a, b, q))
        return True

    def add_uni(q: str) -> bool:
        options = [p for p in split(q) if key((q,), p) not in seen]
        if not options:
            return False
        b, c = options[rng.integers(len(options))]
        seen.add(key((q,), (b, c)))
        uni.append((q, b, c))
        return True

    def add_two(first: str | None = None) -> bool:
        a = first if first is not None else species[rng.integers(len(species))]
        b = species[rng.integers(len(species))]
        s = tuple(x + y for x, y in zip(vec[a], vec[b]))
        options = [p for p in pairs.get(s, []) if sorted(p) != sorted((a, b)) and key((a, b), p) not in seen]
        if not options:
            return False
        c, d = options[rng.integers(len(options))]
        seen.add(key((a, b), (c, d)))
        two.append((a, b, c, d))
        return True

    # every species takes part: molecules by a three-body formation (or a decomposition), atoms by an exchange
    for q in rng.permutation(species):
        q = str(q)
        done = False
        if q in molecules and len(three) + len(low) < n3:
            done = add_three(q)
        if not done and q in molecules and len(uni) < nu:
            done = add_uni(q)
        for _ in range(200):
            if done:
                break
            done = add_two(q)
    tries = 0
    while len(three) + len(low) < n3 and tries < 100000:
        add_three(molecules[rng.integers(len(molecules))])
        tries += 1
    while len(uni) < nu and tries < 200000:
        add_uni(molecules[rng.integers(len(molecules))])
        tries += 1
    while len(two) < n2 and tries < 400000:
        add_two()
        tries += 1
    if len(two) != n2 or len(three) + len(low) != n3 or len(uni) != nu:
        raise RuntimeError(f"could not draw {spec}: {len(two)}, {len(three) + len(low)}, {len(uni)}")

    lines = [f"# Synthetic VULCAN-format network, seed {spec.seed}: {len(species) + 1} species, "
             f"{spec.reactions} reactions, {spec.branches} photolysis branches.",
             "# Stand-in for a real network of the same size; not chemistry for science.", ""]
    rid = 1
    lines.append("# Two-body Reactions")
    lines.append("# id  [ reaction ]  A  B  C")
    for a, b, c, d in two:
        lines.append(f"{rid} [ {a} + {b} -> {c} + {d} ]  {_arrhenius(rng, 1e-16, 1e-9)}")
        rid += 2
    for a, b, c in uni:
        lines.append(f"{rid} [ {a} -> {b} + {c} ]  {_arrhenius(rng, 1e-4, 1e4)}")
        rid += 2
    lines += ["", "# 3-body and Disscoiation Reactions", "# id  [ reaction ]  A_0  B_0  C_0  A_inf  B_inf  C_inf"]
    for a, b, c in three:
        k0 = _arrhenius(rng, 1e-16 / _ND_COLLISION, 1e-9 / _ND_COLLISION)
        kinf = _arrhenius(rng, 1e-12, 1e-9, 1.0, 1e4)
        lines.append(f"{rid} [ {a} + {b} + M -> {c} + M ]  {k0}  {kinf}")
        rid += 2
        if rng.random() < 0.4:
            t = (rng.uniform(0.2, 0.9), rng.uniform(50, 500), rng.uniform(500, 5000), rng.uniform(1000, 8000))
            lines.append(f"Troe [{t[0]:.3f}, {t[1]:.1f}, {t[2]:.1f}, {t[3]:.1f}]")
        if rng.random() < 0.2:
            lines.append(f"effi {{'H2': {rng.uniform(1.0, 3.0):.2f}, 'He': {rng.uniform(0.3, 1.0):.2f}}}")
    lines += ["", "# 3-body reactions without high-pressure rates", "# id  [ reaction ]  A_0  B_0  C_0"]
    for a, b, c in low:
        lines.append(f"{rid} [ {a} + {b} + M -> {c} + M ]  {_arrhenius(rng, 1e-16 / _ND_COLLISION, 1e-9 / _ND_COLLISION)}")
        rid += 2
        if rng.random() < 0.2:
            lines.append(f"effi {{'H2': {rng.uniform(1.0, 3.0):.2f}, 'He': {rng.uniform(0.3, 1.0):.2f}}}")
    if special:
        lines += ["", "# special cases", f"{rid} [ OH + CH3 + M -> CH3OH + M ]"]
        rid += 2
    lines += ["", "# reverse stops", "# photo disscoiation (no reversals)"]
    absorbers = [q for q in molecules if split(q)]
    branch: dict[str, int] = {}
    used: set[Any] = set()
    nb = 0
    while nb < spec.branches:
        q = absorbers[rng.integers(len(absorbers))]
        options = [p for p in split(q) if (q, p) not in used]
        if not options:
            continue
        p = options[rng.integers(len(options))]
        used.add((q, p))
        branch[q] = branch.get(q, 0) + 1
        lines.append(f"{rid} [ {q} -> {p[0]} + {p[1]} ]  {q}  {branch[q]}")
        rid += 2
        nb += 1
    lines += ["", "# condensation", f"{rid} [ H2O -> H2O_l ]", ""]
    return "\n".join(lines), species + ["He"]


def _cache_dir() -> Path:
    root = os.environ.get("MAXICHEM_B200_CACHE")
    return Path(root) if root else _ROOT / "_build" / "networks"


def network_files(name: str, folder: Path | None = None) -> tuple[Path, Path]:
    """Write (once) and return the network file and the NASA-9 folder of a synthetic network."""
    spec = NETWORKS[name]
    rng = np.random.default_rng(spec.seed)
    text, species = _build_text(spec, rng)
    elements = sorted({x for q in species for x in formula(q)})
    thermo = _thermo(species, elements, np.random.default_rng(spec.seed + 1000))
    digest = hashlib.sha256(text.encode() + repr(sorted(thermo.items())).encode()).hexdigest()[:12]
    base = (folder or _cache_dir()) / f"{name}-{digest}"
    net_file, nasa = base / f"{name}_network.txt", base / "NASA9"
    if not net_file.exists():
        nasa.mkdir(parents=True, exist_ok=True)
        for q, (lo, hi) in thermo.items():
            numbers = [*lo[:7], 0.0, *lo[7:], *hi[:7], 0.0, *hi[7:]]
            rows = [" ".join(f"{v:.17e}" for v in numbers[i : i + 5]) for i in range(0, 20, 5)]
            (nasa / f"{q}.txt").write_text("\n".join(rows) + "\n")
        tmp = net_file.with_suffix(".tmp")
        tmp.write_text(text)
        tmp.replace(net_file)
    return net_file, nasa


def network(name: str) -> VulcanNetwork:
    """The synthetic network ``name`` (one of NETWORKS), read through the VULCAN reader."""
    net_file, nasa = network_files(name)
    return VulcanNetwork(net_file, nasa)


def solar_state(net: VulcanNetwork, cells: int, trace: float = 1e-20) -> np.ndarray:
    """Solar-like start [cells, species]: H2/He/H2O/CH4/CO at C/O = 0.5 (N2/NH3, H2S where present), traces at 1e-20."""
    x = np.full(len(net.species), trace)
    major = {"He": 0.145, "H2O": 5.5e-4, "CH4": 2e-4, "CO": 1.5e-4, "N2": 3e-5, "NH3": 5e-5, "H2S": 2.7e-5}
    for q, v in major.items():
        if q in net.species:
            x[net.species.index(q)] = v
    x[net.species.index("H2")] = 0.0
    x[net.species.index("H2")] = 1.0 - x.sum()
    x = x / x.sum()
    return np.tile(x, (cells, 1))


@dataclass
class Workload:
    """One batch of cells: x [B, S], T, P, dt, h [B], J [B, branches] (float64, host)."""

    x: np.ndarray
    T: np.ndarray
    P: np.ndarray
    dt: np.ndarray
    h: np.ndarray
    J: np.ndarray


def column_grid(levels: int, columns: int, rng: np.random.Generator) -> tuple[np.ndarray, np.ndarray]:
    """T, P of a levels x columns grid: log-P levels from 1e-2 to 1e8 dyn cm^-2, T a smooth 400-2200 K profile
    (hotter deeper) shifted per column, plus uniform noise of +-100 K; flattened column-major (levels fastest)."""
    lp = np.linspace(-2.0, 8.0, levels)
    base = 400.0 + 1800.0 / (1.0 + np.exp(-(lp - 3.0) / 1.5))
    shift = 150.0 * np.sin(2 * np.pi * np.arange(columns) / max(columns, 1) + rng.uniform(0, 2 * np.pi))
    T = base[None, :] + shift[:, None] + rng.uniform(-100.0, 100.0, (columns, levels))
    T = np.clip(T, 400.0, 2200.0)
    P = np.tile(10.0**lp, (columns, 1))
    return T.ravel(), P.ravel()


def photolysis_rates(P: np.ndarray, branches: int, rng: np.random.Generator, lit: np.ndarray | None = None) -> np.ndarray:
    """J [B, branches]: log-uniform in 1e-10..1e-3 s^-1 where P < 1e3 dyn cm^-2 (and lit), else 0."""
    J = 10.0 ** rng.uniform(-10.0, -3.0, (len(P), branches))
    on = P < 1e3
    if lit is not None:
        on = on & lit
    return J * on[:, None]


def workload(net: VulcanNetwork, kind: str, cells: int, seed: int = 0) -> Workload:
    """Seeded inputs of one call.

    kind "cfg0": T log-uniform 500-2500 K, P log-uniform 1e-2..1e8, solar start, h 1e-8 s, dt 1e10 s, dark.
    kind "column": the column grid (64 levels), solar start, h 1e-8 s, dt 300 s, upper-layer J.
    kind "uneven": the column grid with the second half of the columns at night (J = 0); ``cold_start`` then turns a
    quarter of the cells of settled states into cold starts.
    """
    rng = np.random.default_rng(seed)
    nj = len(net.photo)
    if kind == "cfg0":
        T = np.exp(rng.uniform(np.log(500.0), np.log(2500.0), cells))
        P = 10.0 ** rng.uniform(-2.0, 8.0, cells)
        dt = np.full(cells, 1e10)
        J = np.zeros((cells, nj))
    elif kind == "column":
        levels = 64
        columns = -(-cells // levels)
        T, P = column_grid(levels, columns, rng)
        T, P = T[:cells], P[:cells]
        dt = np.full(cells, 300.0)
        J = photolysis_rates(P, nj, rng)
    elif kind == "uneven":
        levels = 64
        columns = -(-cells // levels)
        T, P = column_grid(levels, columns, rng)
        T, P = T[:cells], P[:cells]
        dt = np.full(cells, 300.0)
        J = photolysis_rates(P, nj, rng)
        J[np.arange(cells) // levels >= columns // 2] = 0.0  # night side
    else:
        raise ValueError(f"unknown workload kind {kind}")
    return Workload(solar_state(net, cells), T, P, dt, np.full(cells, 1e-8), J)


def cold_start(x: np.ndarray, h: np.ndarray, seed: int = 0, share: float = 0.25, sigma: float = 2.0):
    """A copy of settled states in which every cell of a seeded `share` is a cold start: x multiplied by a log-normal
    factor of width sigma per species and renormalised, h 1e-10 s. Returns x, h and the cold cells' mask."""
    rng = np.random.default_rng(seed)
    x, h = np.array(x, dtype=np.float64), np.array(h, dtype=np.float64)
    cold = rng.random(x.shape[0]) < share
    f = np.exp(sigma * rng.standard_normal((int(cold.sum()), x.shape[1])))
    xc = x[cold] * f
    x[cold] = xc / xc.sum(1, keepdims=True)
    h[cold] = 1e-10
    return x, h, cold
