"""A network's kernel tables: species order, rate laws, S v and Jacobian term lists, and work counts.

The elimination order is the reference's greedy minimum-degree order on the symmetrised Jacobian pattern with ties
to the lower index (imalsky/maxichem ``maxichem/_tables.py:35-50``), so a matrix factored here has the pivots, and so
the rounding, of the reference's factorisation. Its fill (``_tables.py:137-152``) is recorded only for the oracle's
sparse factorisation and for the work counts: the CUDA kernel factors the matrix densely in this order, which gives
the sparse factorisation's bits for finite data (an entry outside the fill stays exactly 0, and fma(-0, u, a) = a).

Rate-law rows and flags follow ``_tables.py:69-106`` and ``_tables.py:169-203`` (ln A, B, C of k0, of the second k0
term and of k_inf, Troe a, T3, T1, T2, efficiency; flags of maxichem/_constants.py:117-129), because the rate
evaluation reads them the same way. The S v and Jacobian term lists are this project's own layout (CSR by row, by
entry), in ascending reaction order.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Any

import numpy as np

from .constants import (
    FALLOFF_KINDS,
    FL_DMU_SHIFT,
    FL_EFF,
    FL_FALLOFF,
    FL_FORWARD_SHIFT,
    FL_REVERSE_SHIFT,
    FL_SECOND_K0,
    FL_THREE_BODY,
    FL_TROE,
    FL_VM11,
    KIND_TWO_BODY,
    MAX_SPECIES,
    THREE_BODY_KINDS,
)
from .network import VulcanNetwork, check_third_body

RATE_COLUMNS = 14  # ln A0, B0, C0, ln A1, B1, C1, ln Ai, Bi, Ci, Troe a, T3, T1, T2, efficiency


def min_degree_order(pattern: set[tuple[int, int]], n: int) -> list[int]:
    """Greedy minimum-degree elimination order of the symmetrised pattern, ties to the lower index."""
    adjacent: list[set[int]] = [set() for _ in range(n)]
    for i, j in pattern:
        if i != j:
            adjacent[i].add(j)
            adjacent[j].add(i)
    remaining = set(range(n))
    order: list[int] = []
    while remaining:
        best = min(remaining, key=lambda q: (len(adjacent[q] & remaining), q))
        order.append(best)
        clique = adjacent[best] & remaining
        for a in clique:
            adjacent[a] |= clique - {a}
        remaining.discard(best)
    return order


def symbolic_fill(pattern: set[tuple[int, int]], n: int) -> set[tuple[int, int]]:
    """The pattern of L + U of an LU without exchanges, in the pattern's own (elimination) indices."""
    filled = set(pattern)
    rows_of: list[set[int]] = [set() for _ in range(n)]  # column k: rows i > k with (i, k)
    cols_of: list[set[int]] = [set() for _ in range(n)]  # row k: columns j > k with (k, j)
    for i, j in filled:
        if i > j:
            rows_of[j].add(i)
        elif j > i:
            cols_of[i].add(j)
    for k in range(n):
        for i in rows_of[k]:
            for j in cols_of[k]:
                if (i, j) not in filled:
                    filled.add((i, j))
                    if i > j:
                        rows_of[j].add(i)
                    elif j > i:
                        cols_of[i].add(j)
    return filled


def rate_law(r: dict[str, Any]) -> tuple[list[float], int]:
    """A thermal reaction's rate row and law flags (the reference's _law, _tables.py:69-106)."""

    def ln(a: float) -> float:
        return float(np.log(a)) if a > 0 else -np.inf

    if r["kind"] == KIND_TWO_BODY:
        k0, k1, ki = (r["A"], r["B"], r["C"]), (0.0, 0.0, 0.0), (1.0, 0.0, 0.0)
    else:
        k0 = (r["A0"], r["B0"], r["C0"])
        k1 = (r["A1"], r["B1"], r["C1"]) if "A1" in r else (0.0, 0.0, 0.0)
        ki = (r["Ai"], r["Bi"], r["Ci"]) if r["kind"] in FALLOFF_KINDS else (1.0, 0.0, 0.0)
    if min(k0[0], k1[0], ki[0]) < 0:
        raise ValueError(f"negative Arrhenius prefactor in {r['eq']}: the kernel takes ln A")
    row = [ln(k0[0]), k0[1], k0[2], ln(k1[0]), k1[1], k1[2], ln(ki[0]), ki[1], ki[2],
           *r.get("troe", (0.0, 1.0, 1.0, 0.0)), r.get("eff", 1.0)]  # fmt: skip
    flags = (
        FL_FALLOFF * (r["kind"] in FALLOFF_KINDS)
        | FL_SECOND_K0 * ("A1" in r)
        | FL_TROE * ("troe" in r)
        | FL_EFF * ("eff" in r)
        | FL_VM11 * (r.get("width") == "vm11")
    )
    return row, flags


@dataclass
class Tables:
    """Everything the CUDA kernels and the oracle read about one network (numpy arrays, host memory)."""

    ns: int
    nr: int  # thermal reactions, then photolysis branches
    nrt: int
    nj: int
    nel: int
    perm: np.ndarray  # int32 [ns]: network species of elimination row i
    rx: np.ndarray  # uint8 [nr, 6]: elimination rows of reactants 0-2 and products 3-5, padding ns
    rc: np.ndarray  # float64 [nr, 14]
    rf: np.ndarray  # int32 [nr]
    nasa: np.ndarray  # float64 [2, ns, 9]: ranges below / above NASA_SPLIT_T, elimination order
    atoms: np.ndarray  # float64 [ns, nel]: network order
    sv_ptr: np.ndarray  # int32 [ns + 1]: row i's S v terms
    sv_term: np.ndarray  # uint32: reaction | coefficient code << 16 (0: +1, 1: -1, 2: +2, 3: -2)
    jac_ptr: np.ndarray  # int32 [entries + 1]
    jac_entry: np.ndarray  # uint32 [entries]: p << 16 | q (elimination rows / columns)
    jac_term: np.ndarray  # uint32: rate index (r forward, nr + r reverse) | code << 12 | a << 16 | b << 24
    fill: np.ndarray  # uint8 [ns, ns]: the pattern of L + U
    has_troe: bool
    has_eff: bool
    flops: dict[str, float] = field(default_factory=dict)
    streams: dict[int, dict[str, np.ndarray]] = field(default_factory=dict)  # per-thread term streams by group size
    stream_groups: tuple[int, int] = (128, 96)  # the group sizes of the call kernel, CTA first
    species: list[str] = field(default_factory=list)
    elements: list[str] = field(default_factory=list)
    photo: bool = False


_CODE = {1.0: 0, -1.0: 1, 2.0: 2, -2.0: 3}


def build(net: VulcanNetwork, photo: bool, warps: int = 4) -> Tables:
    """Build the tables of ``net``; with ``photo`` its photolysis branches follow the thermal reactions. ``warps``:
    the call kernel's warps per cell, which sets the thread groups of the term streams (the sums do not depend on
    it)."""
    reactions = net.reac + (net.photo if photo else [])
    S = np.asarray(net.S, np.float64)
    if photo:
        S = np.hstack([S, np.asarray(net.Sp, np.float64)])
    ns, nr = S.shape
    nrt = len(net.reac)
    reactants = [list(r["re"]) for r in reactions]
    products = [list(r["pr"]) for r in reactions]
    if ns > MAX_SPECIES or max(len(q) for q in reactants + products) > 3 or np.abs(S).max() > 2:
        raise ValueError(
            f"the kernels hold at most {MAX_SPECIES} species, 3 per side and |S| <= 2; this has {ns} species"
        )
    if nr >= 2048:
        raise ValueError(f"the kernels hold fewer than 2048 reactions; this network has {nr}")
    live = [r for r in range(nr) if np.any(S[:, r] != 0)]
    # d v_r / d n_q terms: (sign, rate index, other species of the side) for each occurrence of q on a side
    rate_terms: dict[tuple[int, int], list[tuple[float, int, list[int]]]] = {}
    for r in live:
        sides = [(reactants[r], r, 1.0)] + ([(products[r], nr + r, -1.0)] if r < nrt else [])
        for side, k, sign in sides:
            for m, q in enumerate(side):
                rate_terms.setdefault((r, q), []).append((sign, k, side[:m] + side[m + 1 :]))
    entries: dict[tuple[int, int], list[tuple[float, tuple[int, int]]]] = {}
    for r, q in rate_terms:
        for p in np.flatnonzero(S[:, r]):
            entries.setdefault((int(p), q), []).append((float(S[p, r]), (r, q)))
    pattern = set(entries) | {(i, i) for i in range(ns)}
    perm = min_degree_order(pattern, ns)
    pos = {s: k for k, s in enumerate(perm)}
    fill_set = symbolic_fill({(pos[i], pos[j]) for i, j in pattern}, ns)

    rx = np.full((nr, 6), ns, np.uint8)
    rc = np.zeros((nr, RATE_COLUMNS), np.float64)
    rf = np.zeros(nr, np.int32)
    for j, r in enumerate(reactions):
        if "rev" in r:
            raise ValueError(
                f"reaction {r.get('eq', j)} has an explicit reverse law, which would be ignored: "
                "every reverse comes from NASA-9; remove its 'rev' entry"
            )
        rx[j, : len(reactants[j])] = [pos[q] for q in reactants[j]]
        if j >= nrt:
            continue  # photolysis: kf = J, no reverse
        check_third_body(r["eq"], r["kind"], f"reaction {j}")
        rx[j, 3 : 3 + len(products[j])] = [pos[q] for q in products[j]]
        row, flags = rate_law(r)
        rc[j] = row
        rf[j] = (
            flags
            | FL_THREE_BODY * (r["kind"] in THREE_BODY_KINDS)
            | (len(products[j]) - len(reactants[j]) + 4) << FL_DMU_SHIFT
            | len(reactants[j]) << FL_FORWARD_SHIFT
            | len(products[j]) << FL_REVERSE_SHIFT
        )

    # S v: row i (elimination order) = sum over reactions in ascending order
    sv_ptr, sv_term = [0], []
    for i in range(ns):
        row = S[perm[i]]
        for r in range(nr):
            if row[r] != 0:
                sv_term.append(r | _CODE[float(row[r])] << 16)
        sv_ptr.append(len(sv_term))

    # Jacobian entries (p, q) in elimination positions, row-major; terms in ascending (reaction, occurrence) order
    by_entry: dict[tuple[int, int], list[int]] = {}
    for (p, q), lst in entries.items():
        words = by_entry.setdefault((pos[p], pos[q]), [])
        for c, (r, q_) in sorted(lst, key=lambda t: t[1][0]):
            for sign, k, rest in rate_terms[(r, q_)]:
                ab = [pos[o] for o in rest] + [ns] * (2 - len(rest))
                words.append(k | _CODE[c * sign] << 12 | ab[0] << 16 | ab[1] << 24)
    jac_entry, jac_ptr, jac_term = [], [0], []
    for (p, q) in sorted(by_entry):
        jac_entry.append(p << 16 | q)
        jac_term.extend(by_entry[(p, q)])
        jac_ptr.append(len(jac_term))

    fill = np.zeros((ns, ns), np.uint8)
    for i, j in fill_set:
        fill[i, j] = 1
    atoms = np.asarray(net.atoms, np.float64)
    tab = Tables(
        ns=ns, nr=nr, nrt=nrt, nj=nr - nrt, nel=atoms.shape[1],
        perm=np.array(perm, np.int32), rx=rx, rc=rc, rf=rf,
        nasa=np.stack([np.asarray(net.lo, np.float64)[perm], np.asarray(net.hi, np.float64)[perm]]),
        atoms=atoms,
        sv_ptr=np.array(sv_ptr, np.int32), sv_term=np.array(sv_term, np.uint32),
        jac_ptr=np.array(jac_ptr, np.int32), jac_entry=np.array(jac_entry, np.uint32),
        jac_term=np.array(jac_term, np.uint32), fill=fill,
        has_troe=any("troe" in r for r in reactions), has_eff=any("eff" in r for r in reactions),
        species=list(net.species), elements=list(net.elements), photo=photo,
    )  # fmt: skip
    tab.flops = work_counts(tab)
    tab.stream_groups = stream_groups(warps)
    for threads in tab.stream_groups:
        tab.streams[threads] = thread_streams(tab, threads)
    return tab


def stream_groups(warps: int) -> tuple[int, int]:
    """The thread groups the call kernel streams sums over: its CTA of `warps` warps, and the warps past the first
    (which evaluate F(Y3) while warp 0 solves stage 2)."""
    return (32 * warps, 32 * (warps - 1))


STREAM_GROUPS = stream_groups(4)  # the library's default CTA of 4 warps
SV_END = 1 << 13
J_END = 1 << 14


def _balance(sizes: list[int], threads: int) -> list[list[int]]:
    """Items over threads, longest first onto the least-loaded thread (ties to the lower thread)."""
    lanes: list[list[int]] = [[] for _ in range(threads)]
    load = np.zeros(threads, np.int64)
    for item in sorted(range(len(sizes)), key=lambda q: (-sizes[q], q)):
        t = int(np.argmin(load))
        lanes[t].append(item)
        load[t] += sizes[item]
    return lanes


def sv_pieces(tab: Tables) -> tuple[int, np.ndarray, list[list[int]]]:
    """The S v rows cut into pieces: the piece length P (a property of the network: the terms over 128 threads, at
    least 8), each row's first piece (int32 [ns + 1]) and each piece's terms. Row i's sum is its pieces' sums added in
    order, each piece summed in ascending reaction order from 0; a row with no terms has one empty piece (sum 0)."""
    total = int(len(tab.sv_term))
    P = max(8, -(-total // 128))
    ptr, pieces = [0], []
    for i in range(tab.ns):
        terms = list(range(int(tab.sv_ptr[i]), int(tab.sv_ptr[i + 1])))
        chunks = [terms[c : c + P] for c in range(0, len(terms), P)] or [[]]
        pieces.extend(chunks)
        ptr.append(len(pieces))
    return P, np.array(ptr, np.int32), pieces


def thread_streams(tab: Tables, threads: int) -> dict[str, np.ndarray]:
    """Each thread's S v pieces and Jacobian entries as coalesced word streams (word q of thread t at q * threads + t).

    S v: a thread sums its pieces (sv_pieces) one after the other; a word is the reaction (11 bits; nr is the zero
    padding), the coefficient code << 11 and SV_END on a piece's last term; sv_rows lists the pieces it writes (their
    index into the row-ordered piece list). Jacobian: a thread forms its entries one after the other, each in its term
    order; a word is the rate index | code << 12 | J_END | a << 16 | b << 24, padding rate 2 nr (a zero) with a = b =
    ns; jac_dst lists the dense index p ld + q of its entries, ld = ns | 1. Every sum keeps its order.
    """
    ns, nr = tab.ns, tab.nr
    ld = ns | 1
    _, _, pieces = sv_pieces(tab)
    by_thread = _balance([max(1, len(pc)) for pc in pieces], threads)
    rounds = max(1, max(sum(max(1, len(pieces[i])) for i in its) for its in by_thread))
    nrow = max(1, max(len(its) for its in by_thread))
    sv = np.full((rounds, threads), nr, np.uint16)
    sv_rows = np.zeros((nrow, threads), np.uint16)
    for t, its in enumerate(by_thread):
        q = 0
        for e, i in enumerate(its):
            sv_rows[e, t] = i
            if not pieces[i]:  # a species in no reaction (an inert bath gas): one zero word writes its sum 0
                sv[q, t] = nr | SV_END
                q += 1
            for n, term in enumerate(pieces[i]):
                w = int(tab.sv_term[term])
                sv[q, t] = (w & 0xFFFF) | ((w >> 16) & 3) << 11 | (SV_END if n == len(pieces[i]) - 1 else 0)
                q += 1
    terms = [list(range(tab.jac_ptr[e], tab.jac_ptr[e + 1])) for e in range(len(tab.jac_entry))]
    by_thread = _balance([len(t) for t in terms], threads)
    jrounds = max(1, max(sum(len(terms[e]) for e in its) for its in by_thread))
    jn = max(1, max(len(its) for its in by_thread))
    pad = (2 * nr) | ns << 16 | ns << 24
    jt = np.full((jrounds, threads), pad, np.uint32)
    jd = np.zeros((jn, threads), np.uint16)
    for t, its in enumerate(by_thread):
        q = 0
        for n, e in enumerate(its):
            pq = int(tab.jac_entry[e])
            jd[n, t] = (pq >> 16) * ld + (pq & 0xFFFF)
            for m, term in enumerate(terms[e]):
                w = int(tab.jac_term[term])
                jt[q, t] = (w & 0x3FFF) | (J_END if m == len(terms[e]) - 1 else 0) | (w & 0xFFFF0000)
                q += 1
    return {"sv": sv, "sv_rows": sv_rows, "jt": jt, "jac_dst": jd}


def sv_row_pieces(tab: Tables) -> tuple[int, np.ndarray]:
    """The piece length and each row's first piece, for the kernels and the oracle."""
    P, ptr, _ = sv_pieces(tab)
    return P, ptr


def work_counts(tab: Tables) -> dict[str, float]:
    """Algorithmic floating-point operations of one cell's work, by part (an fma counts 2).

    rhs: n from Y (NS), rates of progress (multiplies and one subtraction per side), S v (2 per term), F and u0 (2 NS).
    jacobian: 3 per term (k n_a n_b and its fma). w: 2 per Jacobian entry plus NS. lu: on the fill pattern, per pivot
    1 reciprocal, a scaling per L entry and 2 per update. solve: 2 per off-diagonal L or U entry plus NS.
    sherman: the rank-one correction of one solve (4 NS). stage: the Rodas3 stage vectors and error (about 20 NS).
    rates: per call, 30 per species (NASA-9) and 40 per thermal reaction (laws, reverse, limit; a transcendental counts 1).
    """
    ns = tab.ns
    rx = tab.rx
    mult = int(np.sum(rx[:, 0:3] != ns) + np.sum(rx[: tab.nrt, 3:6] != ns))
    rhs = ns + mult + tab.nr + 2 * len(tab.sv_term) + 2 * ns
    jac = 3 * len(tab.jac_term)
    w = 2 * len(tab.jac_entry) + ns
    fill = tab.fill.astype(bool)
    lu = 0
    for k in range(ns):
        rows = int(fill[k + 1 :, k].sum())
        cols = int(fill[k, k + 1 :].sum())
        lu += 1 + rows + 2 * rows * cols
    offdiag = int(fill.sum()) - ns
    solve = 2 * offdiag + ns
    fresh = 3 * rhs + jac + w + lu + 5 * solve + 5 * 4 * ns + 20 * ns
    retry = fresh - rhs - jac - w
    return {
        "rhs": float(rhs), "jacobian": float(jac), "w": float(w), "lu": float(lu), "solve": float(solve),
        "fresh_try": float(fresh), "retry": float(retry), "rates": float(30 * ns + 40 * tab.nrt),
        "dense_lu": float(sum(1 + m + 2 * m * m for m in range(ns))),
    }  # fmt: skip
