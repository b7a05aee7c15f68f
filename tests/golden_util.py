"""Rebuild a golden case's input directory from its fixture and parse it."""
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
CASES = ["gyre_sor", "gyre_mg", "gyre_hk83_a4", "channel", "jets", "full", "gyre_dmg", "jets_dmg"]


def load_case(name, tmp):
    from pawsim_b200 import inputs
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    d = os.path.join(str(tmp), name)
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, "params.dat"), "w") as fh:
        fh.write(str(z["param_text"]))
    for key in z.files:
        if key.startswith("in_"):
            z[key].astype("<f8").tofile(os.path.join(d, key[3:]))
    cfg = inputs.read_config(os.path.join(d, "params.dat"))
    return cfg, inputs.load_fields(cfg), z
