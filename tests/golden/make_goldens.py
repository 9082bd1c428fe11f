"""Generate the committed golden fixtures from the reference's own test data.

Run once in a container that has the reference checkout (``python
tests/golden/make_goldens.py /path/to/voronota-ltr``).  It reads the reference's
bench inputs (``benches/data/balls_*.xyzr``, parsed like ``parse_xyzr`` in
src/input/mod.rs:117-143: the last four columns are x y z r) and the centrality golden
(``tests/data/central_golden.tsv``) as text, and writes:

* ``balls_cs_1x1.npy``, ``balls_2zsk.npy``, ``balls_3dlb.npy`` -- (N, 4) float64 x y z r
* ``central_golden.npy`` -- (20, 3) int64 rows (id_a, id_b, central)
* ``assembly_1ctf.pdb1.gz``, ``assembly_1ctf.cif.gz``, ``1ctf_pdb_cells_reference.tsv.gz``,
  ``custom_radii.txt.gz`` -- the reference's file-input test data (tests/data), gzipped,
  for the file front end's end-to-end goldens

The known answers the tests assert (counts and totals) are the numbers the reference's
own tests assert; they are kept in ``goldens.json`` with the file:line they come from.
Nothing at test time reads the reference checkout.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

KNOWN_ANSWERS = {
    "cs_1x1": {
        "source": "tests/cli.rs:104-117; src/tessellation.rs:1010-1015",
        "probe": 2.0, "contacts": 153, "cells": 100,
        "total_contact_area": 3992.55, "total_sas_area": 21979.64, "total_volume": 46419.87,
        "tol": 0.01, "contact_0_1_area": 42.9555, "contact_0_1_arc": 23.2335, "contact_tol": 0.01,
    },
    "cs_1x1_periodic": {
        "source": "tests/cli.rs:119-156",
        "probe": 2.0, "corners": [[0, 0, 0], [200, 250, 300]], "contacts": 189, "cells": 100,
        "total_contact_area": 4812.14, "total_sas_area": 20023.06, "total_volume": 45173.20, "tol": 0.01,
    },
    "2zsk": {"source": "tests/cli.rs:158-165; tests/updateable.rs:287-303", "probe": 1.4,
             "contacts": 23855, "cells": 3545},
    "ring17": {
        "source": "src/tessellation.rs:741-797",
        "probe": 1.0, "contacts": 44, "cells": 17,
        "cell0_sas": 34.8168, "cell0_vol": 29.2302, "cell1_sas": 3.29195, "cell1_vol": 2.48022,
        "cell_tol": 0.01, "contact_0_1_area": 0.747721, "contact_0_1_arc": 0.726907, "c01_tol": 0.001,
        "contact_1_2_area": 5.0216, "c12_tol": 0.01,
    },
    "ring17_periodic": {
        "source": "src/tessellation.rs:1020-1072",
        "probe": 1.0, "corners": [[-1.6, -1.6, -0.6], [1.6, 1.6, 3.1]], "min_contacts_exclusive": 44,
        "cells": 17, "cell0_sas": 3.56578, "cell0_vol": 20.2781, "cell_tol": 0.1,
        "self_contact_0_0_area": 3.36258, "self_tol": 0.01,
    },
    "two_body_groups": {
        "source": "tests/contacts_only.rs:421-442",
        "probe": 1.4, "contacts": 1, "id_a": 1, "id_b": 2, "area": 23.43431770037136, "tol": 1e-6,
    },
    "centrality": {"source": "tests/centrality_golden.rs:12-66; tests/data/central_golden.tsv",
                   "probe": 1.4, "radius": 1.5},
    "file_1ctf_pdb": {"source": "tests/pdb_mmcif.rs:12-43,99-153; tests/test_python.py:303-315",
                      "probe": 1.4, "balls": 492, "balls_without_hetero": 487, "contacts": 3078, "cells": 492,
                      "total_sas_area": 4097.64, "total_contact_area": 10663.91, "tol": 0.01,
                      "per_atom_tol": 0.01},
    "file_1ctf_cif": {"source": "tests/pdb_mmcif.rs:45-97; tests/test_python.py:317-342",
                      "probe": 1.4, "balls": 984, "contacts": 6354, "cells": 984},
    "file_1ctf_custom_radii": {"source": "tests/pdb_mmcif.rs:216-246", "probe": 1.4, "balls": 984,
                               "contacts": 6354, "total_sas_area": 7094.42, "total_contact_area": 21423.54,
                               "tol": 0.01},
    "radii_lookups": {"source": "tests/pdb_mmcif.rs:130-152",
                      "cases": [["ALA", "CA", 1.90], ["ALA", "N", 1.70], ["ALA", "C", 1.75], ["ALA", "O", 1.49],
                                ["ALA", "CB", 1.92], ["ARG", "NH1", 1.62], ["ZN", "ZN", 0.74]]},
}


def parse_xyzr(path):
    rows = []
    with open(path) as f:
        for line in f:
            parts = line.split()
            if len(parts) < 4:
                continue
            try:
                x, y, z, r = (float(v) for v in parts[-4:])
            except ValueError:
                continue
            rows.append((x, y, z, r))
    return np.array(rows, dtype=np.float64)


def main(ref_root):
    for name in ("cs_1x1", "2zsk", "3dlb"):
        arr = parse_xyzr(os.path.join(ref_root, "benches", "data", f"balls_{name}.xyzr"))
        np.save(os.path.join(HERE, f"balls_{name}.npy"), arr)
        print(name, arr.shape)
    rows = []
    with open(os.path.join(ref_root, "tests", "data", "central_golden.tsv")) as f:
        for line in f:
            if line.startswith("#") or not line.strip():
                continue
            a, b, c = line.split()[:3]
            rows.append((int(a), int(b), int(c)))
    np.save(os.path.join(HERE, "central_golden.npy"), np.array(rows, dtype=np.int64))
    import gzip
    for name in ("assembly_1ctf.pdb1", "assembly_1ctf.cif", "1ctf_pdb_cells_reference.tsv", "custom_radii.txt"):
        with open(os.path.join(ref_root, "tests", "data", name), "rb") as f:
            data = f.read()
        with gzip.GzipFile(os.path.join(HERE, name + ".gz"), "wb", mtime=0) as g:
            g.write(data)
        print(name, len(data))
    with open(os.path.join(HERE, "goldens.json"), "w") as f:
        json.dump(KNOWN_ANSWERS, f, indent=1, sort_keys=True)
    print("centrality rows", len(rows))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_goldens.py <path of the voronota-ltr source tree>")
    main(sys.argv[1])
