"""Extract the golden densities of libcntr's FKM Bethe-quench test (libcntr/test/fkm_bethe_quench.cpp,
"Reference calculation for fkm - commit cae14da") from its HDF5 fixture fkm_bethe_quench.h5 into
tests/golden/fkm_bethe_quench.json.

No HDF5 library is installed here, so this script reads the file's structure directly, following
the published HDF5 file format specification: superblock version 0, the root group's symbol table
(version-1 B-tree of group nodes, symbol-table nodes "SNOD", local heap "HEAP" for the names), and
for each dataset its version-1 object header with the dataspace (0x0001), datatype (0x0003) and
data layout (0x0008, contiguous) messages.  That covers this fixture (two 1-d float64 datasets
"den0" and "den1" of nt + 2 = 52 values); anything else raises.

    NESSI_REFERENCE_ROOT=<reference checkout> python tests/golden/make_fkm_golden.py [path/to/fkm_bethe_quench.h5]
"""
import json
import os
import struct
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
# default source: under NESSI_REFERENCE_ROOT, the reference checkout (the directory holding
# libcntr/); a path given as the first argument overrides it
DEFAULT_SRC = os.path.join(os.environ.get("NESSI_REFERENCE_ROOT", "."), "libcntr/test/fkm_bethe_quench.h5")
OUT = os.path.join(HERE, "fkm_bethe_quench.json")
SIGNATURE = b"\x89HDF\r\n\x1a\n"


class H5:
    def __init__(self, data):
        self.d = data
        if data[:8] != SIGNATURE:
            raise ValueError("not an HDF5 file")
        if data[8] != 0:
            raise ValueError("superblock version %d not supported" % data[8])
        self.so, self.sl = data[13], data[14]  # size of offsets / lengths
        if (self.so, self.sl) != (8, 8):
            raise ValueError("only 8-byte offsets and lengths are supported")
        # superblock v0: 24 bytes of versions and sizes, then base, free-space, end-of-file and
        # driver addresses, then the root group's symbol table entry
        self.root = self.entry(24 + 4 * 8)

    def u(self, off, n):
        return int.from_bytes(self.d[off:off + n], "little")

    def entry(self, off):
        """Symbol table entry: link name offset, object header address, cache type, scratch."""
        name_off, header = self.u(off, 8), self.u(off + 8, 8)
        cache = self.u(off + 16, 4)
        scratch = self.d[off + 24:off + 40]
        e = {"name_off": name_off, "header": header, "cache": cache}
        if cache == 1:  # group: B-tree and local heap addresses cached in the scratch pad
            e["btree"], e["heap"] = struct.unpack("<QQ", scratch)
        return e

    def heap_name(self, heap, off):
        if self.d[heap:heap + 4] != b"HEAP":
            raise ValueError("bad local heap")
        data = self.u(heap + 24, 8)
        s = self.d[data + off:]
        return s[:s.index(b"\0")].decode()

    def group_entries(self, g):
        out = []
        stack = [g["btree"]]
        while stack:
            node = stack.pop()
            if self.d[node:node + 4] != b"TREE":
                raise ValueError("bad B-tree node")
            ntype, level, used = self.d[node + 4], self.d[node + 5], self.u(node + 6, 2)
            if ntype != 0:
                raise ValueError("not a group B-tree")
            # keys (heap offsets, 8 bytes) and children alternate after the sibling addresses
            base = node + 8 + 2 * 8
            children = [self.u(base + 8 + i * 16, 8) for i in range(used)]
            if level > 0:
                stack.extend(children)
                continue
            for snod in children:
                if self.d[snod:snod + 4] != b"SNOD":
                    raise ValueError("bad symbol table node")
                n = self.u(snod + 6, 2)
                for i in range(n):
                    e = self.entry(snod + 8 + i * 40)
                    e["name"] = self.heap_name(g["heap"], e["name_off"])
                    out.append(e)
        return out

    def messages(self, header):
        """Messages of a version-1 object header (continuation blocks followed)."""
        if self.d[header] != 1:
            raise ValueError("object header version %d not supported" % self.d[header])
        nmsg, size = self.u(header + 2, 2), self.u(header + 8, 4)
        blocks = [(header + 16, size)]
        out = []
        while blocks and len(out) < nmsg:
            off, size = blocks.pop(0)
            end = off + size
            while off + 8 <= end and len(out) < nmsg:
                mtype, msize = self.u(off, 2), self.u(off + 2, 2)
                body = off + 8
                if mtype == 0x0010:  # continuation
                    blocks.append((self.u(body, 8), self.u(body + 8, 8)))
                out.append((mtype, body, msize))
                off = body + msize
        return out

    def dataset(self, header):
        dims = dtype = layout = None
        for mtype, body, _ in self.messages(header):
            if mtype == 0x0001:  # dataspace, version 1
                ver, rank = self.d[body], self.d[body + 1]
                if ver != 1:
                    raise ValueError("dataspace version %d not supported" % ver)
                dims = [self.u(body + 8 + 8 * i, 8) for i in range(rank)]
            elif mtype == 0x0003:  # datatype
                cls = self.d[body] & 0x0F
                size = self.u(body + 4, 4)
                bits = self.d[body + 1]
                if cls != 1 or size != 8 or (bits & 1):
                    raise ValueError("only little-endian float64 datasets are supported")
                dtype = "<d"
            elif mtype == 0x0008:  # data layout
                ver, cls = self.d[body], self.d[body + 1]
                if ver != 3 or cls != 1:
                    raise ValueError("only contiguous layout (version 3) is supported")
                layout = (self.u(body + 2, 8), self.u(body + 10, 8))
        if dims is None or dtype is None or layout is None:
            raise ValueError("dataset messages missing")
        n = 1
        for x in dims:
            n *= x
        addr, nbytes = layout
        if nbytes != 8 * n:
            raise ValueError("layout size %d does not match %d values" % (nbytes, n))
        return list(struct.unpack("<%dd" % n, self.d[addr:addr + nbytes]))


def main(src):
    f = H5(open(src, "rb").read())
    data = {e["name"]: f.dataset(e["header"]) for e in f.group_entries(f.root)}
    out = {"source": "libcntr/test/fkm_bethe_quench.h5 (read by tests/golden/make_fkm_golden.py)",
           "test": "libcntr/test/fkm_bethe_quench.cpp: nt=50, ntau=200, beta=5, h=0.01, U0=1, U1=2, order 5",
           "den0": data["den0"], "den1": data["den1"]}
    with open(OUT, "w") as fh:
        json.dump(out, fh, indent=1)
    print("wrote", OUT, {k: len(v) for k, v in data.items()})


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else DEFAULT_SRC)
