#!/usr/bin/env python3
"""Copy the reference's own example configurations (data/examples_fmo/ of
noma/dm-heom: the FMO complex at 77 K for population dynamics, linear
absorption and circular dichroism) into tests/golden/fmo/, with only
solver.steps reduced so that a GPU test and the oracle finish in seconds.
Every other line is kept as the reference ships it.

Usage: python make_fmo_fixtures.py [REFERENCE_ROOT]
       (default: $HEOM_REFERENCE_ROOT, else /root/reference)
"""
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
STEPS = {"fmo_population_dynamics_77K.cfg": 100,
         "fmo_linear_absorption_77K.cfg": 50,
         "fmo_circular_dichroism_77K.cfg": 50}


def main():
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("HEOM_REFERENCE_ROOT", "/root/reference")
    src_dir = os.path.join(root, "data", "examples_fmo")
    out_dir = os.path.join(HERE, "fmo")
    os.makedirs(out_dir, exist_ok=True)
    for name, steps in STEPS.items():
        text = open(os.path.join(src_dir, name)).read()
        new, n = re.subn(r"(?m)^steps=\d+$", f"steps={steps}", text)
        assert n == 1, name
        header = (f"# {name} of noma/dm-heom (data/examples_fmo/), solver.steps reduced to {steps} "
                  f"by tests/golden/make_fmo_fixtures.py; nothing else changed\n")
        with open(os.path.join(out_dir, name), "w") as f:
            f.write(header + new)
        print("wrote", os.path.join(out_dir, name))


if __name__ == "__main__":
    main()
