"""The VULCAN reader against the reference reader's results (golden), and its refusals."""

import json
from pathlib import Path

import numpy as np
import pytest

import invented
from maxichem_b200 import synthetic
from maxichem_b200.network import VulcanNetwork

GOLDEN = Path(__file__).parent / "golden"


@pytest.fixture(scope="module")
def golden():
    return json.loads((GOLDEN / "reader.json").read_text()), np.load(GOLDEN / "reader.npz")


def _plain(r):
    return json.loads(json.dumps({k: (list(v) if isinstance(v, tuple) else v) for k, v in r.items()}))


@pytest.mark.parametrize("name", list(synthetic.NETWORKS))
def test_synthetic_network_reads_as_the_reference_reads_it(golden, networks, name):
    meta, arrays = golden
    net = networks(name)
    ref = meta[name]
    assert net.species == ref["species"] and net.elements == ref["elements"]
    assert net.skipped == ref["skipped"] and net.photo_missing == ref["photo_missing"]
    assert [list(d) for d in net.duplicates] == ref["duplicates"]
    for key in ("S", "Sp", "atoms", "lo", "hi"):
        assert np.array_equal(getattr(net, key), arrays[f"{name}/{key}"]), key
    assert [_plain(r) for r in net.reac] == ref["reac"]
    assert [_plain(r) for r in net.photo] == ref["photo"]


def test_network_sizes_are_the_configs():
    sizes = {n: (len(s.species) + 1, s.reactions, s.branches) for n, s in synthetic.NETWORKS.items()}
    assert sizes == {"cho41": (41, 207, 36), "chno69": (69, 390, 48), "sncho91": (91, 532, 61)}


def _net(tmp_path, text, species=("A", "B", "He")):
    thermo = {q: invented.constant_cp(0.0) for q in species}
    return invented.write(tmp_path, text, thermo)


@pytest.mark.parametrize(
    "text,match",
    [
        ("# Two-body Reactions\n1 [ H2 + O -> H2O + H ] 1 0 0\n", "do not balance"),
        ("1 [ H + O -> OH ] 1 0 0\n", "above the first heading"),
        ("# Two-body Reactions\n# bogus heading\n1 [ H + OH -> H2 + O ] 1 0 0\n", "unknown heading"),
        ("# irreversible\n1 [ H + OH -> H2 + O ] 1 0 0\n", "irreversible"),
        ("# Two-body Reactions\n1 [ H + OH -> H2 + O ] nan 0 0\n", "finite rate coefficients"),
        ("# Two-body Reactions\n1 [ H + OH -> H2 + O ] 1 0\n", "3 rate coefficients"),
        ("# Two-body Reactions\n1 [ H + OH + M -> H2 + O + M ] 1 0 0\n", "law needs M on neither"),
        ("# 3-body reactions without high-pressure rates\n1 [ H + H -> H2 ] 1 0 0\n", "law needs M on both"),
        ("# Two-body Reactions\n1 [ H + OH -> H2 + O ] 1 0 0\n# reverse stops\n3 [ H + OH -> H2 + O ] 1 0 0\n",
         "outside photolysis"),
        ("# Two-body Reactions\n1 [ H + OH -> H2 + O ] 1 0 0\n# reverse stops\n# photo\n3 [ OH -> O + H ] H2O 1\n",
         "not its absorber"),
        ("# Two-body Reactions\n1 [ H + OH -> H2 + O ] 1 0 0\nTroe [1, 2, 3]\n", "4 numbers"),
        ("# Two-body Reactions\n1 [ H + OH -> H2 + O ] 1 0 0\neffi {'He': 2}\n", "bulk gas"),
        ("# special cases\n1 [ H + OH + M -> H2O + M ]\n", "unknown special"),
    ],
)
def test_malformed_networks_are_refused(tmp_path, text, match):
    thermo = {q: invented.constant_cp(0.0) for q in ("H", "O", "OH", "H2", "H2O", "He")}
    with pytest.raises(ValueError, match=match):
        invented.write(tmp_path, text, thermo)


def test_nasa9_ranges_that_do_not_meet_are_refused(tmp_path):
    text = "# Two-body Reactions\n1 [ CO_1 + He -> CO_2 + He ] 1e-11 0 0\n"
    thermo = {"CO_1": (invented.constant_cp(0.0), invented.constant_cp(50.0)), "CO_2": invented.constant_cp(0.0),
              "He": invented.constant_cp(0.0)}  # fmt: skip
    with pytest.raises(ValueError, match="jumps"):
        invented.write(tmp_path, text, thermo)


def test_missing_nasa9_file_is_refused(tmp_path):
    text = "# Two-body Reactions\n1 [ CO_1 + He -> CO_2 + He ] 1e-11 0 0\n"
    net_file = tmp_path / "n.txt"
    net_file.write_text(text)
    (tmp_path / "NASA9").mkdir()
    with pytest.raises(FileNotFoundError, match="no NASA-9 file"):
        VulcanNetwork(net_file, tmp_path / "NASA9")


def test_species_order_and_repeats(tmp_path):
    net = invented.write(tmp_path, invented.ISOMERS, {q: invented.constant_cp(0.0) for q in ("CO_1", "CO_2", "He")})
    assert net.species == ["CO_1", "He", "CO_2"]  # first appearance; He already named
    with pytest.raises(ValueError, match="more than once"):
        VulcanNetwork(tmp_path / "network.txt", tmp_path / "NASA9", species=["CO_1", "CO_1", "CO_2", "He"])


def test_condensation_lines_are_counted_whatever_their_form(tmp_path):
    text = ("# Two-body Reactions\n1 [ H + OH -> H2 + O ] 1 0 0\n# reverse stops\n# condensation\n"
            "5 [ H2O -> H2O_l_s ] 1 2\n6 [ not a reaction ]\n")  # fmt: skip
    thermo = {q: invented.constant_cp(0.0) for q in ("H", "O", "OH", "H2", "He")}
    assert invented.write(tmp_path, text, thermo).skipped == 2
