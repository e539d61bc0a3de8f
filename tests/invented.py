"""Small invented networks for the known-answer tests, written in VULCAN's format with NASA-9 files of constant Cp.

Not chemistry for science: each network isolates one law or one answer that is known without the solver.
"""

from pathlib import Path

import numpy as np

from maxichem_b200.network import VulcanNetwork

BOLTZMANN = 1.380649e-16  # erg K^-1, typed here so a wrong solver constant cannot also move an answer
STANDARD_PRESSURE = 1.0e6  # dyn cm^-2


def constant_cp(h_over_r: float, cp: float = 3.5, s_over_r: float = 0.0) -> list[float]:
    """One NASA-9 range a1..a7, b1, b2 with Cp/R = cp, H/R = cp T + h_over_r, S/R = cp ln T + s_over_r."""
    return [0.0, 0.0, cp, 0.0, 0.0, 0.0, 0.0, h_over_r, s_over_r]


def gibbs_rt(a, T: float) -> float:
    """G/RT of one NASA-9 range (McBride et al. 2002), written out."""
    lt = np.log(T)
    h = -a[0] / T**2 + a[1] * lt / T + a[2] + a[3] * T / 2 + a[4] * T**2 / 3 + a[5] * T**3 / 4 + a[6] * T**4 / 5
    s = -a[0] / T**2 / 2 - a[1] / T + a[2] * lt + a[3] * T + a[4] * T**2 / 2 + a[5] * T**3 / 3 + a[6] * T**4 / 4
    return float((h + a[7] / T) - (s + a[8]))


def write(folder: Path, text: str, thermo: dict) -> VulcanNetwork:
    """Write a network and its NASA-9 files (one range for both sides of 1000 K, or a (low, high) pair)."""
    nasa = Path(folder) / "NASA9"
    nasa.mkdir(parents=True, exist_ok=True)
    for name, ranges in thermo.items():
        low, high = ranges if isinstance(ranges, tuple) else (ranges, ranges)
        numbers = [*low[:7], 0.0, *low[7:], *high[:7], 0.0, *high[7:]]
        rows = [" ".join(f"{q:.17e}" for q in numbers[i : i + 5]) for i in range(0, 20, 5)]
        (nasa / f"{name}.txt").write_text("\n".join(rows) + "\n")
    (Path(folder) / "network.txt").write_text(text)
    return VulcanNetwork(Path(folder) / "network.txt", nasa)


def state(net: VulcanNetwork, cells: int, **fractions: float) -> np.ndarray:
    x = np.zeros((cells, len(net.species)))
    for name, v in fractions.items():
        x[:, net.species.index(name)] = v
    return x / x.sum(1, keepdims=True)


DECAY = """# Invented: A -> 2 B by photolysis; the thermal row of zero rate names the species
# Two-body Reactions
1 [ N2_1 + N_1 -> N_1 + N2_1 ] 0.0 0.0 0.0

# reverse stops
# photo disscoiation (no reversals)
3 [ N2_1 -> N_1 + N_1 ] N2_1 1
"""


def decay(folder: Path) -> VulcanNetwork:
    thermo = {q: constant_cp(0.0) for q in ("N2_1", "N_1")} | {"He": constant_cp(0.0, 2.5)}
    return write(folder, DECAY, thermo)


def decay_answer(jt):
    """Mole fractions of A and B for A -> 2 B at constant pressure from pure A: N_A = e^-Jt, N_B = 2 (1 - e^-Jt)."""
    a = np.exp(-np.asarray(jt))
    return a / (2.0 - a), 2.0 * (1.0 - a) / (2.0 - a)


RECOMBINATION = """# Invented: H + H + M -> H2 + M with a negligible reverse
# 3-body reactions without high-pressure rates
1 [ H + H + M -> H2 + M ] 1.0E-32 0.0 0.0

# reverse stops
"""
RECOMBINATION_K0 = 1.0e-32
RECOMBINATION_T = 1000.0


def recombination(folder: Path):
    atom = constant_cp(0.0, 2.5)
    thermo = {"H": atom, "H2": constant_cp(-2.0e5), "He": atom}
    return write(folder, RECOMBINATION, thermo), thermo


def recombination_time(n, P: float):
    """t at which N_H = n from pure H: dN/dt = -2 k0 nd^2 N^2 / sum N with sum N = (1 + N) / 2, so
    1/N - ln N = 1 + 4 k0 nd^2 t at constant pressure."""
    nd = P / (BOLTZMANN * RECOMBINATION_T)
    return (1.0 / np.asarray(n) - np.log(n) - 1.0) / (4.0 * RECOMBINATION_K0 * nd**2)


ISOMERS = """# Invented: two isomers exchanging on collisions with He
# Two-body Reactions
1 [ CO_1 + He -> CO_2 + He ] 1e-11 0 0
"""

HYDROGEN = """# Invented: hydrogen-oxygen exchanges with NASA-9 equilibria
# Two-body Reactions
1 [ H + OH -> H2 + O ] 1.0E-11 0.0 1000.0
3 [ H + H2O -> OH + H2 ] 1.0E-11 0.0 2000.0

# 3-body reactions without high-pressure rates
5 [ H + H + M -> H2 + M ] 2.7E-31 -0.6 0.0

# reverse stops
"""


def hydrogen(folder: Path):
    thermo = {
        "H": constant_cp(26000.0, 2.5, 14.0), "OH": constant_cp(4500.0, 3.5, 21.0),
        "H2": constant_cp(0.0, 3.5, 15.0), "O": constant_cp(30000.0, 2.5, 18.0),
        "H2O": constant_cp(-29000.0, 4.0, 20.0), "He": constant_cp(0.0, 2.5, 15.0),
    }  # fmt: skip
    return write(folder, HYDROGEN, thermo), thermo
