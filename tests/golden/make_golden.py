"""Write the golden fixtures of tests/golden from the reference implementation (imalsky/maxichem).

Run where the reference is checked out (read-only is enough), with its path as the one argument; the fixtures it
writes are committed, so the tests never need the reference itself:

  python tests/golden/make_golden.py /path/to/reference

* reader.json / reader.npz: the reference reader's VulcanNetwork of each synthetic network (species, elements,
  S, Sp, atoms, NASA-9 ranges, reaction dicts);
* tables.npz: the reference table builder's elimination order, fill (leading part), rate rows, flags and species
  slots of each synthetic network, with and without photolysis;
* rates.npz: forward and reverse rate coefficients of each synthetic network's thermal reactions at a grid of (T, P),
  from the reference tests' own written-out laws (tests/test_rate_laws.py arrhenius, falloff, troe_factor;
  tests/helpers.py gibbs_rt) and the collision rule of docs/method.md;
* dense_lu.npz: matrices and their threshold-pivoted factors by the reference test's rule (tests/test_dense_lu.py
  threshold_lu);
* first_trial.json: one Rodas3 step of A -> 2 B from (1, 0), exactly, by the reference test's rational arithmetic
  (tests/test_known_answers.py _first_trial).
"""

from __future__ import annotations

import json
import sys
from fractions import Fraction
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
if len(sys.argv) != 2 or not (Path(sys.argv[1]) / "maxichem").is_dir():
    sys.exit("usage: python tests/golden/make_golden.py /path/to/reference  (a checkout of imalsky/maxichem)")
REFERENCE = Path(sys.argv[1])
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(REFERENCE))
sys.path.insert(0, str(REFERENCE / "tests"))

import helpers  # noqa: E402  (the reference's test helpers)
import test_dense_lu  # noqa: E402
import test_known_answers  # noqa: E402
import test_rate_laws  # noqa: E402
from maxichem import _constants, _tables, kinvulcan  # noqa: E402

from maxichem_b200 import synthetic  # noqa: E402

CONDITIONS = [(500.0, 1e-2), (800.0, 1e3), (1200.0, 1e6), (1800.0, 1e7), (2500.0, 1e8)]


def _jsonable(r: dict) -> dict:
    out = {}
    for k, v in r.items():
        if isinstance(v, tuple):
            v = list(v)
        if k == "names":
            v = [list(q) for q in v]
        out[k] = v
    return out


def reader_and_tables() -> None:
    meta, arrays, tabs = {}, {}, {}
    for name in synthetic.NETWORKS:
        f, nasa = synthetic.network_files(name)
        net = kinvulcan.VulcanNetwork(f, nasa)
        meta[name] = {
            "species": net.species, "elements": net.elements, "skipped": net.skipped,
            "duplicates": [list(d) for d in net.duplicates], "photo_missing": net.photo_missing,
            "reac": [_jsonable(r) for r in net.reac], "photo": [_jsonable(r) for r in net.photo],
        }  # fmt: skip
        for key in ("S", "Sp", "atoms", "lo", "hi"):
            arrays[f"{name}/{key}"] = np.asarray(getattr(net, key))
        for photo in (False, True):
            tab = _tables.tables(net, 2, photo)
            k0 = tab["k0"]
            lead = np.array(sorted(e for e in tab["pattern"] if not (e[0] >= k0 and e[1] >= k0)), np.int32)
            p = f"{name}/{int(photo)}"
            tabs[f"{p}/perm"] = tab["perm"]
            tabs[f"{p}/lead"] = lead
            tabs[f"{p}/k0"] = np.array(k0)
            tabs[f"{p}/rc"] = tab["rc"]
            tabs[f"{p}/rf"] = tab["rf"]
            tabs[f"{p}/rx"] = tab["rx"]
    (HERE / "reader.json").write_text(json.dumps(meta))
    np.savez_compressed(HERE / "reader.npz", **arrays)
    np.savez_compressed(HERE / "tables.npz", **tabs)


def _law_k(r: dict, T: float, nd: float) -> float:
    """k of a thermal reaction from the reference tests' written-out laws (M not folded in)."""
    if r["kind"] == _constants.KIND_TWO_BODY:
        k = test_rate_laws.arrhenius(r["A"], r["B"], r["C"], T)
    else:
        k0 = test_rate_laws.arrhenius(r["A0"], r["B0"], r["C0"], T)
        if "A1" in r:
            k0 += test_rate_laws.arrhenius(r["A1"], r["B1"], r["C1"], T)
        if r["kind"] in _constants.FALLOFF_KINDS:
            kinf = test_rate_laws.arrhenius(r["Ai"], r["Bi"], r["Ci"], T)
            troe = r.get("troe")
            k = test_rate_laws.falloff(k0, kinf, nd, T, troe, vm11=r.get("width") == "vm11") if k0 > 0 else 0.0
        else:
            k = k0
    return k * r.get("eff", 1.0)


def rates() -> None:
    out = {}
    for name in synthetic.NETWORKS:
        f, nasa = synthetic.network_files(name)
        net = kinvulcan.VulcanNetwork(f, nasa)
        kf_all, kr_all = [], []
        for T, P in CONDITIONS:
            nd = float(helpers.number_density(T, P))
            g = [helpers.gibbs_rt(net.lo[i] if T < 1000.0 else net.hi[i], T) for i in range(len(net.species))]
            kfs, krs = [], []
            for r in net.reac:
                k = _law_k(r, T, nd)
                three = r["kind"] in _constants.THREE_BODY_KINDS
                dg = sum(g[q] for q in r["pr"]) - sum(g[q] for q in r["re"])
                dmu = len(r["pr"]) - len(r["re"])
                kf = k * (nd if three else 1.0)
                kr = k * np.exp(dg + dmu * np.log(helpers.BOLTZMANN * T / helpers.STANDARD_PRESSURE)) * (
                    nd if three else 1.0
                )
                # docs/method.md, collision limit: q = k n_tot^(b + m - 2) with k without M, where m + b >= 2
                b = 1 if three else 0
                q = 0.0
                for m, kk in ((len(r["re"]), kf), (len(r["pr"]), kr)):
                    if m + b >= 2:
                        q = max(q, kk / (nd if three else 1.0) * nd ** (b + m - 2))
                if q > _constants.K_COLL:
                    kf, kr = kf * _constants.K_COLL / q, kr * _constants.K_COLL / q
                kfs.append(kf)
                krs.append(kr)
            kf_all.append(kfs)
            kr_all.append(krs)
        out[f"{name}/kf"] = np.array(kf_all)
        out[f"{name}/kr"] = np.array(kr_all)
    out["conditions"] = np.array(CONDITIONS)
    np.savez_compressed(HERE / "rates.npz", **out)


def dense_lu() -> None:
    rng = np.random.default_rng(11)
    mats = test_dense_lu._matrices(42, rng)
    out = {"a": mats}
    factors, orders, ex = [], [], []
    for m in mats:
        order, f, exchanges, kept = test_dense_lu.threshold_lu(m)
        factors.append(f)
        orders.append(order)
        ex.append((exchanges, kept))
    out.update(factors=np.array(factors), orders=np.array(orders), exchanges=np.array(ex))
    np.savez_compressed(HERE / "dense_lu.npz", **out)


def first_trial() -> None:
    z = Fraction(1, 10)
    new, k4 = test_known_answers._first_trial(z)
    (HERE / "first_trial.json").write_text(
        json.dumps({"z": [z.numerator, z.denominator], "new": [[q.numerator, q.denominator] for q in new],
                    "k4": [[q.numerator, q.denominator] for q in k4]})  # fmt: skip
    )


if __name__ == "__main__":
    reader_and_tables()
    rates()
    dense_lu()
    first_trial()
    for p in sorted(HERE.iterdir()):
        print(p.name, p.stat().st_size)
