"""Fixtures read from the reference's test files by make_fixtures.py (committed JSON)."""
import json
import os

_HERE = os.path.dirname(os.path.abspath(__file__))


def load(name):
    with open(os.path.join(_HERE, name + ".json")) as f:
        return json.load(f)
