"""File front end (voronota_ltr.io) on the CPU: parsing, radii, selections and groupings
against the reference's file-input tests (tests/pdb_mmcif.rs, src/input/*.rs unit tests,
tests/test_python.py:296-382), with the tessellation of the parsed balls by the oracle
pinned to the reference's end-to-end goldens (counts, totals, the C++ per-atom cells)."""
import gzip
import os

import numpy as np
import pytest

import oracle as O
from common import GOLDEN, goldens
from voronota_ltr import io as VIO

G = goldens()
PDB = os.path.join(GOLDEN, "assembly_1ctf.pdb1.gz")
CIF = os.path.join(GOLDEN, "assembly_1ctf.cif.gz")


def reference_cells():
    with gzip.open(os.path.join(GOLDEN, "1ctf_pdb_cells_reference.tsv.gz"), "rt") as f:
        rows = [l.rstrip("\n").split("\t") for l in f.readlines()[1:]]
    rows = [r for r in rows if len(r) >= 8]
    return (np.array([int(r[5]) for r in rows]), np.array([float(r[6]) for r in rows]),
            np.array([float(r[7]) for r in rows]))


def test_parse_counts():  # tests/pdb_mmcif.rs:12-23,45-62,80-128
    g = G["file_1ctf_pdb"]
    assert len(VIO.parse_file(PDB).balls) == g["balls"]
    assert len(VIO.parse_file(PDB, VIO.ParseOptions(exclude_heteroatoms=True)).balls) == g["balls_without_hetero"]
    cif = VIO.parse_file(CIF)
    assert len(cif.balls) == G["file_1ctf_cif"]["balls"]
    assert sorted({r.chain_id for r in cif.records}) == ["A", "A-2"]
    asm = VIO.parse_file(PDB, VIO.ParseOptions(as_assembly=True))
    assert len(asm.balls) == len(cif.balls)
    assert sorted({r.chain_id for r in asm.records}) == ["A", "A2"]


def test_radii_lookups():  # tests/pdb_mmcif.rs:130-152; radii.rs tests
    R = VIO.RadiiLookup.default()
    for res, atom, r in G["radii_lookups"]["cases"]:
        assert abs(R.radius(res, atom) - r) < 1e-3
    assert R.radius("XYZ", "") == 1.8 and R.radius("XYZ", "*") == 1.8
    assert R.radius("UNK", "QQ") == 1.8  # no rule
    assert R.radius("UNK", "CX9") == 1.80 and R.radius("UNK", "NZZ") == 1.60  # prefix rules
    E = VIO.RadiiLookup()
    E.load_text("# c\n*  *  2.5\nALA CB 1.0\n")
    assert E.radius("ALA", "CB") == 1.0 and E.radius("GLY", "N") == 2.5
    for bad in ("ALA CB", "ALA CB x", "ALA CB -1"):
        with pytest.raises(ValueError):
            VIO.RadiiLookup().load_text(bad)


def test_pdb_columns_and_filters():  # pdb.rs parse_atom_line / is_acceptable
    lines = [
        "ATOM      1  N   MET A   1       0.000   0.000   0.000  1.00  0.00           N",
        "ATOM      2 1HB  MET A   1       1.000   0.000   0.000  1.00  0.00           H",
        "ATOM      3  CA AMET A   1       1.458   0.000   0.000  1.00  0.00           C",
        "ATOM      4  CA BMET A   1       1.500   0.000   0.000  1.00  0.00           C",
        "HETATM    5  O   HOH A 200       9.000   9.000   9.000  1.00  0.00           O",
        "HETATM   99  ZN  ZN  A 100       5.000   5.000   5.000  1.00 12.50          ZN",
        "ENDMDL",
        "ATOM      6  C   MET A   1       2.009   1.420   0.000  1.00  0.00           C",
    ]
    recs = VIO.parse_pdb(lines)
    assert [r.name for r in recs] == ["N", "CA", "ZN"]  # H, altloc B, water dropped; model 2 ignored
    assert recs[1].alt_loc == "" and recs[2].b_factor == 12.5 and recs[2].record_name == "HETATM"
    with_h = VIO.parse_pdb(lines, VIO.ParseOptions(include_hydrogens=True))
    assert [r.name for r in with_h][:2] == ["N", "HB1"]  # leading digit rotated
    asm = VIO.parse_pdb(lines, VIO.ParseOptions(as_assembly=True))
    assert asm[-1].chain_id == "A2"


def test_mmcif_tokens_and_models():  # mmcif.rs
    text = """data_x
loop_
_atom_site.group_PDB
_atom_site.id
_atom_site.label_atom_id
_atom_site.label_comp_id
_atom_site.label_asym_id
_atom_site.label_seq_id
_atom_site.Cartn_x
_atom_site.Cartn_y
_atom_site.Cartn_z
_atom_site.type_symbol
_atom_site.pdbx_PDB_model_num
ATOM 1 N MET A 1 0.0 0.0 0.0 N 1
ATOM 2 "C A" MET A 1 1.0 0.0 0.0 C 1  # a comment
ATOM 3 O ? A 1 2.0 0.0 0.0 O 2
loop_
_other.x
1
"""
    recs = VIO.parse_mmcif(text.splitlines())
    assert [r.name for r in recs] == ["N", "C A"] and recs[0].res_name == "MET"
    asm = VIO.parse_mmcif(text.splitlines(), VIO.ParseOptions(as_assembly=True))
    assert len(asm) == 3 and asm[2].chain_id == "A2" and asm[2].res_name == ""


def test_format_detection_and_xyzr(tmp_path):  # mod.rs:80-143
    assert VIO.detect_format("a.PDB", None) == "pdb" and VIO.detect_format("a.ent", None) == "pdb"
    assert VIO.detect_format("a.mmcif", None) == "mmcif" and VIO.detect_format("a.xyzr", None) == "xyzr"
    assert VIO.detect_format("a.txt", "data_1abc") == "mmcif"
    assert VIO.detect_format("a.txt", "HEADER    x") == "pdb"
    assert VIO.detect_format("a.txt", "at 1 2 3 4") == "xyzr"
    assert VIO.detect_format("a.txt", "hello") is None
    p = tmp_path / "b.dat"
    p.write_text("1.0 2.0 3.0 4.0\nx 5.0 6.0 7.0 8.0\nbad line\n")
    s = VIO.parse_file(str(p))
    assert s.balls.tolist() == [[1.0, 2.0, 3.0, 4.0], [5.0, 6.0, 7.0, 8.0]] and s.records == []
    q = tmp_path / "c.dat"
    q.write_text("nothing here\n")
    with pytest.raises(OSError):
        VIO.parse_file(str(q))


def test_selections():  # selection.rs
    def rec(chain="A", res="ALA", seq=5, name="CA", kind="ATOM"):
        return VIO.AtomRecord(kind, 1, name, "", res, chain, seq, "", 0.0, 0.0, 0.0, "C")

    S = VIO.Selection
    assert S("chain A").matches(rec()) and not S("chain B").matches(rec())
    assert S("chain A-2").matches(rec(chain="A-2")) and not S("chain A-2").matches(rec())
    assert S("resname AL?").matches(rec()) and S("resname [A-C]LA").matches(rec())
    assert S("resid 1 to 9").matches(rec()) and S("resid 5").matches(rec()) and not S("resid 6:9").matches(rec())
    assert S("resid -3 to 5").matches(rec()) and S("resid 1:9").matches(rec())
    assert S("protein and backbone").matches(rec()) and not S("sidechain").matches(rec())
    assert S("not (chain B or resname GLY)").matches(rec())
    assert S("hetatm").matches(rec(kind="HETATM")) and S("charged").matches(rec(res="LYS"))
    assert S("name 'C*'").matches(rec()) and S("all") .matches(rec()) and not S("none").matches(rec())
    for bad in ("", "chain", "resid", "and chain A", "(chain A", "chain A )", "foo A", "resid 1 to", "chain A $"):
        with pytest.raises(VIO.SelectionError):
            S(bad)
    assert VIO.glob_match("*", "") and VIO.glob_match("A*B", "AxxB") and not VIO.glob_match("A*B", "AxxC")
    groups = VIO.build_custom_grouping([rec(chain="A"), rec(chain="B"), rec(chain="C"), rec(chain="C")],
                                       VIO.parse_selections(["chain A", "chain B"]))
    assert groups.tolist() == [0, 1, 2, 3]
    with pytest.raises(VIO.SelectionError):
        VIO.parse_selections(["chain A"])
    recs = [rec(chain="A", seq=1), rec(chain="A", seq=2), rec(chain="B", seq=1), rec(chain="A", seq=1)]
    assert VIO.build_chain_grouping(recs).tolist() == [0, 0, 1, 0]
    assert VIO.build_residue_grouping(recs).tolist() == [0, 1, 2, 0]


def test_oracle_on_parsed_files():  # tests/pdb_mmcif.rs:26-43,64-78,155-246
    g = G["file_1ctf_pdb"]
    balls = VIO.parse_file(PDB).balls
    o = O.compute(balls, g["probe"])
    assert (len(o.contacts_a), len(o.cells_index)) == (g["contacts"], g["cells"])
    assert abs(o.total_sas_area - g["total_sas_area"]) < g["tol"]
    assert abs(o.total_contact_area - g["total_contact_area"]) < g["tol"]
    idx, sas, vol = reference_cells()  # the C++ voronota per-atom cells
    assert np.array_equal(o.cells_index.astype(np.int64), idx)
    assert np.abs(o.cells_sas - sas).max() < g["per_atom_tol"] and np.abs(o.cells_vol - vol).max() < g["per_atom_tol"]
    assert len(O.compute(VIO.parse_file(CIF).balls, 1.4).contacts_a) == G["file_1ctf_cif"]["contacts"]
    gc = G["file_1ctf_custom_radii"]
    R = VIO.RadiiLookup()
    with gzip.open(os.path.join(GOLDEN, "custom_radii.txt.gz"), "rt") as f:
        R.load_text(f.read())
    b = VIO.parse_file(PDB, VIO.ParseOptions(as_assembly=True), R).balls
    o = O.compute(b, gc["probe"])
    assert (len(b), len(o.contacts_a)) == (gc["balls"], gc["contacts"])
    assert abs(o.total_sas_area - gc["total_sas_area"]) < gc["tol"]
    assert abs(o.total_contact_area - gc["total_contact_area"]) < gc["tol"]


def test_from_file_errors_without_device(tmp_path):  # tests/test_python.py:359-382
    with pytest.raises(IOError):
        VIO.compute_tessellation_from_file(str(tmp_path / "nonexistent.pdb"), 1.4)
    with pytest.raises(IOError):
        VIO.compute_tessellation_from_file(PDB, 1.4, group_selections=["protein"])
    x = tmp_path / "a.xyzr"
    x.write_text("0 0 0 1.5\n3 0 0 1.5\n")
    with pytest.raises(IOError):
        VIO.compute_tessellation_from_file(str(x), 1.4, group_selections=["chain A", "chain B"])
    with pytest.raises(IOError):
        VIO.compute_tessellation_from_file(PDB, 1.4, group_selections=["chain A", "bogus X"])
