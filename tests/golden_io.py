"""Reads the golden fixtures written by tests/golden/make_golden.py."""
import hashlib
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def cases():
    with open(os.path.join(GOLDEN, "manifest.json")) as f:
        return json.load(f)["cases"]


def load(case):
    x = np.load(os.path.join(GOLDEN, case["name"] + ".in.npy"))
    with open(os.path.join(GOLDEN, case["name"] + ".sleek"), "rb") as f:
        s = f.read()
    return x, s


def sha(b) -> str:
    return hashlib.sha256(bytes(b)).hexdigest()
