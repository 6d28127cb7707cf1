"""Loader for the golden QuickPar vectors in tests/golden/quickpar.json."""
import base64
import hashlib
import json
import os
import struct
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
        self.packets = []
        for p in doc.get("par2_packets", []):
            hdr = bytes.fromhex(p["header"])
            if "exponent" in p:
                body = struct.pack("<I", p["exponent"]) + self.recovery[p["exponent"]].tobytes()
            else:
                body = _unpack(p["body"])
            self.packets.append((hdr, body))
        self.par2_files = doc.get("par2_files", [])

    def par2_bytes(self, name):
        """The QuickPar .par2 file `name`, rebuilt byte for byte."""
        for f in self.par2_files:
            if f["name"] == name:
                buf = b"".join(self.packets[i][0] + self.packets[i][1] for i in f["packets"])
                assert len(buf) == f["size"] and hashlib.md5(buf).hexdigest() == f["md5"]
                return buf
        raise KeyError(name)

    def materialize(self, d):
        """Writes the data files and the seven .par2 files of the set into d."""
        for f in self.files:
            with open(os.path.join(d, f["name"]), "wb") as o:
                o.write(f["data"])
        for f in self.par2_files:
            with open(os.path.join(d, f["name"]), "wb") as o:
                o.write(self.par2_bytes(f["name"]))
        return d

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
