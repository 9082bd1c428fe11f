"""compute_tessellation_from_file end to end on the GPU (tests/test_python.py:296-382,
tests/pdb_mmcif.rs): the reference's counts and totals, and the C++ per-atom cells of
1ctf within 0.01, in both precisions."""
import gzip
import os

import numpy as np
import pytest

import oracle as O
import voronota_ltr as V
from common import GOLDEN, goldens
from gpu_util import compare
from test_io_cpu import CIF, PDB, reference_cells
from voronota_ltr import io as VIO

pytestmark = pytest.mark.gpu
G = goldens()
PRECISIONS = ["fp64", "fp32"]


@pytest.mark.parametrize("prec", PRECISIONS)
def test_pdb_file(prec):
    g = G["file_1ctf_pdb"]
    d = V.compute_tessellation_from_file(PDB, probe=1.4, precision=prec)
    assert d["num_balls"] == g["balls"] and len(d["contacts"]) == g["contacts"] and len(d["cells"]) == g["cells"]
    assert abs(d["total_sas_area"] - g["total_sas_area"]) < g["tol"]
    assert abs(d["total_contact_area"] - g["total_contact_area"]) < g["tol"]
    idx, sas, vol = reference_cells()
    assert [c["index"] for c in d["cells"]] == idx.tolist()
    assert np.abs(np.array([c["sas_area"] for c in d["cells"]]) - sas).max() < g["per_atom_tol"]
    assert np.abs(np.array([c["volume"] for c in d["cells"]]) - vol).max() < g["per_atom_tol"]
    balls = VIO.parse_file(PDB).balls
    compare(V.compute_tessellation_result(balls, 1.4, precision=prec), O.compute(balls, 1.4), prec)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_mmcif_file_and_selections(prec):
    g = G["file_1ctf_cif"]
    d = V.compute_tessellation_from_file(CIF, probe=1.4, precision=prec)
    assert d["num_balls"] == g["balls"] and len(d["contacts"]) == g["contacts"] and len(d["cells"]) == g["cells"]
    s = V.compute_tessellation_from_file(CIF, probe=1.4, group_selections=["chain A", "chain A-2"], precision=prec)
    assert 0 < len(s["contacts"]) < g["contacts"]
    parsed = VIO.parse_file(CIF)
    groups = VIO.build_custom_grouping(parsed.records, VIO.parse_selections(["chain A", "chain A-2"]))
    compare(V.compute_tessellation_result(parsed.balls, 1.4, groups=groups, precision=prec),
            O.compute(parsed.balls, 1.4, groups=groups), prec)
    for c in s["contacts"]:  # inter-chain contacts only
        assert parsed.records[c["id_a"]].chain_id != parsed.records[c["id_b"]].chain_id


def test_with_cell_vertices_and_custom_radii():
    d = V.compute_tessellation_from_file(PDB, probe=1.4, with_cell_vertices=True)
    assert "cell_vertices" in d and "cell_edges" in d and len(d["cell_vertices"]) > 0
    gc = G["file_1ctf_custom_radii"]
    R = VIO.RadiiLookup()
    with gzip.open(os.path.join(GOLDEN, "custom_radii.txt.gz"), "rt") as f:
        R.load_text(f.read())
    d = V.compute_tessellation_from_file(PDB, 1.4, radii=R, options=VIO.ParseOptions(as_assembly=True))
    assert d["num_balls"] == gc["balls"] and len(d["contacts"]) == gc["contacts"]
    assert abs(d["total_sas_area"] - gc["total_sas_area"]) < gc["tol"]
    assert abs(d["total_contact_area"] - gc["total_contact_area"]) < gc["tol"]
