"""Extracts the golden vectors in tests/golden/quickpar.json from the QuickPar
fixture set that par2-rs bundles (tests/data/testdata*.par2 and
tests/data/test-*.data in the par2-rs repository).

Run where the par2-rs sources are available, giving their fixture folder:

    python tests/golden/make_golden.py <par2-rs checkout>/tests/data

The output holds, in the canonical input-slice order of the set (the order of
the Main packet's recovery-set File ID list, as par2-rs parser.rs:522-596
establishes it):

  * the slice size and every file's name, length and contents (zlib+base64);
  * every file's IFSC entries (MD5, CRC32 of each zero-padded slice);
  * every recovery slice: exponent and body (zlib+base64);
  * every distinct packet of the .par2 files (its 64-byte header and, except
    for RecvSlic packets, whose body is the recovery slice above behind its
    4-byte exponent, its body) and every .par2 file as the list of its packets
    in file order, so that a test can rebuild each file byte for byte
    (checked here against the file) and compare the packets a writer produces
    header by header.

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


def packet_list(buf):
    """(offset, header, type, body) of every valid packet, in file order."""
    pos, out = 0, []
    for ptype, body in packets(buf):
        pos = buf.find(MAGIC, pos)
        while hashlib.md5(buf[pos + 32:pos + 64] + buf[pos + 64:pos + 64 + len(body)]).digest() \
                != buf[pos + 16:pos + 32]:
            pos = buf.find(MAGIC, pos + 1)
        out.append((pos, buf[pos:pos + 64], ptype, body))
        pos += 64 + len(body)
    return out


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
    par2_files, unique, index = [], [], {}
    for path in sorted(glob.glob(os.path.join(src_dir, "testdata*.par2"))):
        buf = open(path, "rb").read()
        plist, rebuilt = [], b""
        for off, hdr, ptype, body in packet_list(buf):
            assert off == len(rebuilt), (path, off)  # packets are contiguous
            if hdr not in index:  # the header's MD5 covers the body
                ent = {"header": hdr.hex()}
                if ptype == T_RECV:
                    (exp,) = struct.unpack_from("<I", body, 0)
                    assert body[4:] == recv[exp]
                    ent["exponent"] = exp
                else:
                    ent["body"] = pack(body)
                index[hdr] = len(unique)
                unique.append(ent)
            plist.append(index[hdr])
            rebuilt += hdr + body
        assert rebuilt == buf, path
        par2_files.append({"name": os.path.basename(path), "size": len(buf),
                           "md5": hashlib.md5(buf).hexdigest(), "packets": plist})
    doc = {"source": "par2-rs tests/data (QuickPar 0.4 set testdata.par2 + volumes)",
           "block_size": block_size, "files": files, "recovery": recovery,
           "par2_packets": unique, "par2_files": par2_files}
    with open(out_path, "w") as f:
        json.dump(doc, f, indent=1)
    print(f"wrote {out_path}: block_size={block_size} files={len(files)} "
          f"slices={sum(len(f['ifsc']) for f in files)} recovery={len(recovery)} "
          f"par2 files={len(par2_files)}")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <par2-rs checkout>/tests/data")
    main(sys.argv[1], os.path.join(os.path.dirname(os.path.abspath(__file__)), "quickpar.json"))
