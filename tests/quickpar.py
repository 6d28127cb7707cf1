"""Loader for the golden QuickPar vectors in tests/golden/quickpar.json."""
import base64
import json
import os
import zlib

import numpy as np

_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "quickpar.json")


def _unpack(s):
    return zlib.decompress(base64.b64decode(s))


class QuickParSet:
    def __init__(self):
        doc = json.load(open(_PATH))
        self.block_size = doc["block_size"]
        self.files = []
        for f in doc["files"]:
            self.files.append(dict(f, data=_unpack(f["data"])))
        self.recovery = {r["exponent"]: np.frombuffer(_unpack(r["body"]), np.uint8)
                         for r in doc["recovery"]}
        self.recovery_md5 = {r["exponent"]: r["md5"] for r in doc["recovery"]}

    def slices(self, files=None):
        """Zero-padded input slices in canonical order: uint8 [k, block_size],
        plus per-slice (file index, slice-in-file)."""
        bs = self.block_size
        out, owner = [], []
        for fi, f in enumerate(self.files):
            data = f["data"]
            n = (len(data) + bs - 1) // bs
            for b in range(n):
                chunk = data[b * bs:(b + 1) * bs]
                out.append(np.frombuffer(chunk.ljust(bs, b"\x00"), np.uint8))
                owner.append((fi, b))
        return np.stack(out), owner

    def file_index(self, name):
        for i, f in enumerate(self.files):
            if f["name"] == name:
                return i
        raise KeyError(name)

    def slice_base(self, name):
        """Global index of the first slice of file `name`."""
        base = 0
        for f in self.files:
            if f["name"] == name:
                return base
            base += (len(f["data"]) + self.block_size - 1) // self.block_size
        raise KeyError(name)


def load():
    return QuickParSet()
