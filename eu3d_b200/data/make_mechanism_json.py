"""Regenerate h2_ja919.json from an EU3D checkout's input files.

    python -m eu3d_b200.data.make_mechanism_json /path/to/EU3D/input

The JSON holds the tables that Reaction::ReactionRead builds from
H2_JA919.txt and thermo.dat (parsed by eu3d_b200.readers, which restates that
reader), so that benchmarks and tests run where the input files are absent.
"""
import json
import os
import sys

from eu3d_b200.readers import read_mechanism


def main(input_dir: str, out: str = os.path.join(os.path.dirname(os.path.abspath(__file__)), "h2_ja919.json")):
    mech = read_mechanism(os.path.join(input_dir, "H2_JA919.txt"), os.path.join(input_dir, "thermo.dat"))
    with open(out, "w") as fh:
        json.dump(mech.to_json(), fh, indent=1)
    print(out)


if __name__ == "__main__":
    main(sys.argv[1])
