"""Extracts the golden vectors in tests/golden/quickpar.json from the QuickPar
fixture set that par2-rs bundles (tests/data/testdata*.par2 and
tests/data/test-*.data in the par2-rs repository).

Run in a container that has the par2-rs sources mounted:

    python tests/golden/make_golden.py /root/reference/tests/data

The output holds, in the canonical input-slice order of the set (the order of
the Main packet's recovery-set File ID list, as par2-rs parser.rs:522-596
establishes it):

  * the slice size and every file's name, length and contents (zlib+base64);
  * every file's IFSC entries (MD5, CRC32 of each zero-padded slice);
  * every recovery slice: exponent and body (zlib+base64).

Packets are parsed with the PAR2 header layout of par2-rs writer.rs:92-123
(magic, u64 length, packet MD5 over set-id+type+body, set id, type, body) and
every packet's MD5 is checked before it is used.  Nothing here is needed at
test time: the tests read only the JSON.
"""
import base64
import glob
import hashlib
import json
import os
import struct
import sys
import zlib

MAGIC = b"PAR2\x00PKT"
T_MAIN = b"PAR 2.0\x00Main\x00\x00\x00\x00"
T_DESC = b"PAR 2.0\x00FileDesc"
T_IFSC = b"PAR 2.0\x00IFSC\x00\x00\x00\x00"
T_RECV = b"PAR 2.0\x00RecvSlic"


def packets(buf):
    pos = 0
    while True:
        pos = buf.find(MAGIC, pos)
        if pos < 0 or pos + 64 > len(buf):
            return
        (length,) = struct.unpack_from("<Q", buf, pos + 8)
        if length < 64 or pos + length > len(buf):
            pos += 1
            continue
        md5 = buf[pos + 16:pos + 32]
        setid = buf[pos + 32:pos + 48]
        ptype = buf[pos + 48:pos + 64]
        body = buf[pos + 64:pos + length]
        if hashlib.md5(setid + ptype + body).digest() != md5:
            pos += 1
            continue
        yield ptype, body
        pos += length


def pack(b):
    return base64.b64encode(zlib.compress(bytes(b), 9)).decode()


def main(src_dir, out_path):
    main_order = None
    block_size = None
    desc = {}
    ifsc = {}
    recv = {}
    for path in sorted(glob.glob(os.path.join(src_dir, "testdata*.par2"))):
        for ptype, body in packets(open(path, "rb").read()):
            if ptype == T_MAIN:
                block_size, nfiles = struct.unpack_from("<QI", body, 0)
                main_order = [body[12 + 16 * i:28 + 16 * i] for i in range(nfiles)]
            elif ptype == T_DESC:
                fid = body[:16]
                (length,) = struct.unpack_from("<Q", body, 48)
                name = body[56:].split(b"\x00")[0].decode()
                desc[fid] = {"name": name, "length": length,
                             "md5": body[16:32].hex(), "md5_16k": body[32:48].hex()}
            elif ptype == T_IFSC:
                fid = body[:16]
                ents = []
                for o in range(16, len(body), 20):
                    ents.append([body[o:o + 16].hex(), struct.unpack_from("<I", body, o + 16)[0]])
                ifsc[fid] = ents
            elif ptype == T_RECV:
                (exp,) = struct.unpack_from("<I", body, 0)
                recv[exp] = body[4:]
    files = []
    for fid in main_order:
        d = desc[fid]
        data = open(os.path.join(src_dir, d["name"]), "rb").read()
        assert len(data) == d["length"]
        files.append({"file_id": fid.hex(), "name": d["name"], "length": d["length"],
                      "md5": d["md5"], "md5_16k": d["md5_16k"],
                      "ifsc": ifsc[fid], "data": pack(data)})
    recovery = [{"exponent": e, "body": pack(recv[e]),
                 "md5": hashlib.md5(recv[e]).hexdigest()} for e in sorted(recv)]
    doc = {"source": "par2-rs tests/data (QuickPar 0.4 set testdata.par2 + volumes)",
           "block_size": block_size, "files": files, "recovery": recovery}
    with open(out_path, "w") as f:
        json.dump(doc, f, indent=1)
    print(f"wrote {out_path}: block_size={block_size} files={len(files)} "
          f"slices={sum(len(f['ifsc']) for f in files)} recovery={len(recovery)}")


if __name__ == "__main__":
    src = sys.argv[1] if len(sys.argv) > 1 else "/root/reference/tests/data"
    main(src, os.path.join(os.path.dirname(os.path.abspath(__file__)), "quickpar.json"))
