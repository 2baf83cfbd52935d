"""Loaders of the golden vectors restated from the reference's unit tests
(tests/golden/make_exchange_fixtures.py)."""
import json
import os

import numpy as np

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


class Fixtures:
    def __init__(self):
        with open(os.path.join(GOLD, "exchange_fixtures.json")) as f:
            self.cases = json.load(f)["cases"]
        self._npz = np.load(os.path.join(GOLD, "exchange_fixtures.npz"))
        with open(os.path.join(GOLD, "layout_tables.json")) as f:
            self.tables = json.load(f)

    def flat(self, key):
        return self._npz[key].astype(np.int64)

    def array(self, key, shape, layout):
        """A stored memory image as a logical array of `shape`."""
        return self.flat(key).reshape(shape, order="C" if layout == "right" else "F")

    def per_rank(self, key, nprocs, shape, layout):
        """Concatenated per-rank buffers of one shape, rank by rank."""
        a = self.flat(key)
        n = int(np.prod(shape))
        order = "C" if layout == "right" else "F"
        return [a[r * n:(r + 1) * n].reshape(shape, order=order) for r in range(nprocs)]

    def of_kind(self, kind):
        return [c for c in self.cases if c["kind"] == kind]


def distribute_extents(n, r, p):
    base, rem = divmod(n, p)
    return r * base + min(r, rem), base + (1 if r < rem else 0)
