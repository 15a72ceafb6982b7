"""Writes upf_reference_pins.json: what ``inq_b200.pseudo.read_upf`` parses from the pseudopotential
files of the reference's unit-test data (N.upf, N_non_diagonal.upf.gz, F.UPF) -- element, valence
charge, angular momenta of the radial projectors, D_ij in Hartree and the projector radius.

The CPU tests build the KB coefficients from these values and compare them with the numbers the
reference's projector test asserts (projector.hpp:160-240), so the pin holds where the reference tree
is absent; with INQ_REFERENCE_DATA pointing at the data directory they also re-parse the files.

Run from the repository root:  python tests/golden/make_upf_golden.py <data_dir>
(data_dir: the reference's share/unit_tests_data; INQ_REFERENCE_DATA is used when no argument is given)
"""

import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from inq_b200 import pseudo  # noqa: E402

FILES = ["N.upf", "N_non_diagonal.upf.gz", "F.UPF"]


def main():
    data = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("INQ_REFERENCE_DATA")
    if not data:
        sys.exit("usage: make_upf_golden.py <reference share/unit_tests_data directory> "
                 "(or set INQ_REFERENCE_DATA)")
    out = {}
    for name in FILES:
        ps = pseudo.read_upf(os.path.join(data, name))
        out[name] = {"element": ps.element, "z_valence": ps.z_valence, "beta_l": list(ps.beta_l),
                     "dij": ps.dij.tolist(), "projector_radius": ps.projector_radius(), "mesh_size": int(len(ps.r))}
    with open(os.path.join(HERE, "upf_reference_pins.json"), "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    main()
