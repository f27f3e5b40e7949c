"""Loader for tests/golden/ref_collectives.npz (outputs of the reference)."""
import json
import os

import numpy as np

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_ref_collectives():
    z = np.load(os.path.join(HERE, "ref_collectives.npz"))
    index = json.loads(bytes(z["index"]).decode())
    cases = []
    for i, c in enumerate(index):
        c = dict(c)
        if c["ok"]:
            c["out"] = z[f"out{i}"]
            c["msgs"] = z[f"msg{i}"]
        cases.append(c)
    return cases


def load_json(name):
    with open(os.path.join(HERE, name)) as f:
        return json.load(f)
