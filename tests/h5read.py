"""A small HDF5 reader for the tests, written from the HDF5 file format
specification (version 0/1 superblocks, after a user block or not, version 1
object headers, symbol-table groups, contiguous layouts (layout messages
versions 1 to 3) and compact ones, fixed-point, floating point, fixed-length
and variable-length string types, version 1/2 dataspaces, version 1
attributes, global heap collections).

It is the checker of the library's HDF5 writer: besides reading the content
back it asserts the structural rules a conforming reader relies on (the
signatures, the end-of-file address, object header message counts and
sizes, symbol-table nodes sorted by name, B-tree keys bracketing the names
of their children, local heap and global heap bounds).  No part of it is
shared with the writer.
"""
from __future__ import annotations

import struct

import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF
SIG = b"\x89HDF\r\n\x1a\n"


class Dataset:
    def __init__(self, value, attrs, dtype_desc):
        self.value = value
        self.attrs = attrs
        self.dtype_desc = dtype_desc


class H5Read:
    def __init__(self, path):
        with open(path, "rb") as f:
            raw = f.read()
        self.gcol_cache = {}
        # the superblock sits at 0, 512, 1024, 2048, ... (after a user block)
        at = 0
        while raw[at:at + 8] != SIG:
            at = 512 if at == 0 else 2 * at
            assert at < len(raw), "superblock signature"
        b = raw[at:]
        ver = b[8]
        assert ver in (0, 1), f"superblock version {ver}"
        self.so, self.sl = b[13], b[14]
        assert (self.so, self.sl) == (8, 8), "8-byte offsets and lengths"
        self.leaf_k, self.node_k = struct.unpack_from("<HH", b, 16)
        p = 24 + (4 if ver == 1 else 0)
        base, _free, eof, _drv = struct.unpack_from("<4Q", b, p)
        assert base == at, "addresses are relative to the superblock"
        # the stored end-of-file address counts the bytes before the base
        assert eof == len(raw), f"end-of-file address {eof} vs size {len(raw)}"
        self.b, self.eof = b, eof - base
        p += 32
        _name_off, root_oh, cache, _ = struct.unpack_from("<QQII", b, p)
        scratch = struct.unpack_from("<QQ", b, p + 24)
        self.root_oh = root_oh
        self.root_scratch = scratch if cache == 1 else None

    # ---- low level
    def u(self, fmt, off):
        return struct.unpack_from("<" + fmt, self.b, off)

    def check_addr(self, a, n=1):
        assert a != UNDEF and a + n <= self.eof, f"address {a}+{n} beyond end of file"

    # ---- object headers
    def messages(self, addr):
        self.check_addr(addr, 16)
        ver, _, nmsg, _refc, size = self.u("BBHII", addr)
        assert ver == 1, f"object header version {ver}"
        msgs = []
        chunks = [(addr + 16, size)]
        while chunks:
            p, n = chunks.pop(0)
            assert n % 8 == 0
            self.check_addr(p, n)
            end = p + n
            while p < end:
                assert p + 8 <= end
                t, sz, flags = self.u("HHB", p)
                assert sz % 8 == 0, "message data is padded to 8 bytes"
                data = self.b[p + 8:p + 8 + sz]
                assert p + 8 + sz <= end, "message runs past its chunk"
                if t == 0x0010:  # continuation
                    caddr, clen = struct.unpack_from("<QQ", data)
                    chunks.append((caddr, clen))
                msgs.append((t, flags, data))
                p += 8 + sz
        assert len(msgs) == nmsg, f"object header says {nmsg} messages, holds {len(msgs)}"
        return msgs

    # ---- datatypes / dataspaces
    def datatype(self, d, off=0):
        """(description dict, encoded size)"""
        cv = d[off]
        cls, ver = cv & 0x0F, cv >> 4
        assert ver in (1, 2, 3)
        bf = d[off + 1] | (d[off + 2] << 8) | (d[off + 3] << 16)
        size = struct.unpack_from("<I", d, off + 4)[0]
        p = off + 8
        if cls == 0:
            assert bf & 1 == 0, "little-endian"
            bit_off, prec = struct.unpack_from("<HH", d, p)
            return {"class": "int", "size": size, "signed": bool(bf & 8),
                    "bit_offset": bit_off, "precision": prec}, 12
        if cls == 1:
            assert bf & 1 == 0
            bit_off, prec, eloc, esz, mloc, msz, bias = struct.unpack_from("<HHBBBBI", d, p)
            return {"class": "float", "size": size, "norm": (bf >> 4) & 3,
                    "sign": (bf >> 8) & 0xFF, "precision": prec, "exp_loc": eloc,
                    "exp_size": esz, "mant_loc": mloc, "mant_size": msz, "bias": bias}, 20
        if cls == 3:
            return {"class": "string", "size": size, "pad": bf & 0xF, "cset": (bf >> 4) & 0xF}, 8
        if cls == 9:
            base, blen = self.datatype(d, p)
            return {"class": "vlen", "size": size, "kind": bf & 0xF, "pad": (bf >> 4) & 0xF,
                    "cset": (bf >> 8) & 0xF, "base": base}, 8 + blen
        raise AssertionError(f"datatype class {cls} not handled")

    def dataspace(self, d):
        ver, rank, flags = d[0], d[1], d[2]
        if ver == 1:
            p = 8
        else:
            assert ver == 2
            p = 4
            if d[3] == 0:
                return ()
        dims = struct.unpack_from(f"<{rank}Q", d, p)
        return tuple(dims)

    # ---- heaps
    def local_heap(self, addr):
        self.check_addr(addr, 32)
        assert self.b[addr:addr + 4] == b"HEAP", "local heap signature"
        assert self.b[addr + 4] == 0
        seg_size, free_head, seg_addr = self.u("QQQ", addr + 8)
        self.check_addr(seg_addr, seg_size)
        seg = self.b[seg_addr:seg_addr + seg_size]
        assert free_head == 1 or free_head < seg_size, "free-list head"
        assert seg[0] == 0, "offset 0 of a group's heap is the empty name"
        return seg

    def heap_name(self, seg, off):
        assert off < len(seg)
        end = seg.index(b"\0", off)
        return seg[off:end].decode()

    def global_heap(self, addr):
        if addr in self.gcol_cache:
            return self.gcol_cache[addr]
        self.check_addr(addr, 16)
        assert self.b[addr:addr + 4] == b"GCOL", "global heap signature"
        assert self.b[addr + 4] == 1
        size = self.u("Q", addr + 8)[0]
        assert size >= 4096 and size % 8 == 0
        self.check_addr(addr, size)
        objs, p, end = {}, addr + 16, addr + size
        while p < end:
            if p + 16 > end:
                break
            idx, _refc, _res, osz = self.u("HHIQ", p)
            if idx == 0:
                assert p + osz == end, "free space object ends the collection"
                break
            assert idx not in objs
            objs[idx] = self.b[p + 16:p + 16 + osz]
            p += 16 + ((osz + 7) & ~7)
            assert p <= end
        self.gcol_cache[addr] = objs
        return objs

    # ---- values
    def decode(self, dt, shape, raw):
        n = int(np.prod(shape)) if shape else 1
        if dt["class"] == "int":
            assert dt["bit_offset"] == 0 and dt["precision"] == 8 * dt["size"]
            code = {1: "b", 2: "h", 4: "i", 8: "q"}[dt["size"]]
            code = code if dt["signed"] else code.upper()
            a = np.frombuffer(raw, "<" + code, count=n)
        elif dt["class"] == "float":
            assert (dt["size"], dt["precision"], dt["exp_loc"], dt["exp_size"], dt["mant_loc"],
                    dt["mant_size"], dt["bias"], dt["sign"], dt["norm"]) in (
                (8, 64, 52, 11, 0, 52, 1023, 63, 2), (4, 32, 23, 8, 0, 23, 127, 31, 2))
            a = np.frombuffer(raw, "<f8" if dt["size"] == 8 else "<f4", count=n)
        elif dt["class"] == "vlen" and dt["kind"] == 1:
            out = []
            for i in range(n):
                ln, col, idx = struct.unpack_from("<IQI", raw, 16 * i)
                obj = self.global_heap(col)[idx]
                assert len(obj) == ln
                out.append(obj.decode("ascii"))
            return out[0] if not shape else out
        elif dt["class"] == "string":
            s = raw[:dt["size"]]
            return s.split(b"\0", 1)[0].decode("ascii")
        else:
            raise AssertionError(f"no decoder for {dt}")
        return a.reshape(shape) if shape else a[0]

    # ---- objects
    def obj(self, addr):
        msgs = self.messages(addr)
        types = {t for t, _, _ in msgs}
        if 0x0011 in types:
            d = next(d for t, _, d in msgs if t == 0x0011)
            bt, hp = struct.unpack_from("<QQ", d)
            return self.group(bt, hp)
        dt = shape = layout = None
        attrs = {}
        for t, _, d in msgs:
            if t == 0x0001:
                shape = self.dataspace(d)
            elif t == 0x0003:
                dt, _ = self.datatype(d)
            elif t == 0x0008:
                layout = d
            elif t == 0x000C:
                name, val = self.attribute(d)
                attrs[name] = val
        assert dt is not None and shape is not None and layout is not None
        ver = layout[0]
        n = int(np.prod(shape)) if shape else 1
        if ver == 3:
            cls = layout[1]
            if cls == 1:
                a, sz = struct.unpack_from("<QQ", layout, 2)
                assert sz == n * dt["size"], "contiguous size = elements x element size"
            else:
                assert cls == 0
                sz = struct.unpack_from("<H", layout, 2)[0]
                raw = layout[4:4 + sz]
        else:  # versions 1 and 2: rank (+1 for the element size), class, 5 reserved
            assert ver in (1, 2)
            nd, cls = layout[1], layout[2]
            assert cls == 1, "contiguous"
            a = struct.unpack_from("<Q", layout, 8)[0]
            dims = struct.unpack_from(f"<{nd}I", layout, 16)
            sz = int(np.prod(dims))
            assert sz == n * dt["size"]
        if cls == 1:
            self.check_addr(a, sz)
            raw = self.b[a:a + sz]
        return Dataset(self.decode(dt, shape, raw), attrs, dt)

    def attribute(self, d):
        ver = d[0]
        assert ver == 1, f"attribute version {ver}"
        nlen, dtlen, dslen = struct.unpack_from("<HHH", d, 2)
        p = 8
        name = d[p:p + nlen - 1].decode()
        assert d[p + nlen - 1] == 0
        p += (nlen + 7) & ~7
        dt, used = self.datatype(d, p)
        assert used == dtlen
        p += (dtlen + 7) & ~7
        shape = self.dataspace(d[p:p + dslen])
        p += (dslen + 7) & ~7
        n = int(np.prod(shape)) if shape else 1
        return name, self.decode(dt, shape, d[p:p + n * dt["size"]])

    def group(self, btree, heap):
        seg = self.local_heap(heap)
        entries = []
        self.walk(btree, seg, entries, None, None, expect_level=None)
        names = [e[0] for e in entries]
        assert names == sorted(names, key=lambda s: s.encode()), "names in order"
        assert len(set(names)) == len(names)
        out = {}
        for name, oh, cache, scratch in entries:
            o = self.obj(oh)
            if cache == 1:
                assert isinstance(o, dict)
            out[name] = o
        return out

    def walk(self, addr, seg, out, lo, hi, expect_level):
        """Appends the (name, header, cache, scratch) entries under the
        B-tree node at addr, checking that every name lies in (lo, hi]."""
        self.check_addr(addr, 24)
        assert self.b[addr:addr + 4] == b"TREE", "B-tree signature"
        ntype, level, used = self.u("BBH", addr + 4)
        assert ntype == 0, "group B-tree"
        if expect_level is not None:
            assert level == expect_level
        left, right = self.u("QQ", addr + 8)
        assert used <= 2 * self.node_k
        self.check_addr(addr, 24 + (2 * self.node_k + 1) * 8 + 2 * self.node_k * 8)
        p = addr + 24
        keys, kids = [], []
        for i in range(used):
            keys.append(self.u("Q", p)[0])
            kids.append(self.u("Q", p + 8)[0])
            p += 16
        keys.append(self.u("Q", p)[0])
        knames = [self.heap_name(seg, k) for k in keys]
        for i, c in enumerate(kids):
            klo, khi = knames[i], knames[i + 1]
            start = len(out)
            if level > 0:
                self.walk(c, seg, out, klo, khi, level - 1)
            else:
                self.snod(c, seg, out)
            for e in out[start:]:
                assert e[0].encode() > klo.encode() and e[0].encode() <= khi.encode(), \
                    f"name {e[0]!r} outside its keys ({klo!r}, {khi!r}]"
            if out[start:]:
                assert out[-1][0] == khi, "right key is the last name under the child"

    def snod(self, addr, seg, out):
        size = 8 + 2 * self.leaf_k * 40
        self.check_addr(addr, size)
        assert self.b[addr:addr + 4] == b"SNOD", "symbol-table node signature"
        assert self.b[addr + 4] == 1
        n = self.u("H", addr + 6)[0]
        assert 0 < n <= 2 * self.leaf_k
        for i in range(n):
            e = addr + 8 + 40 * i
            off, oh, cache, _ = self.u("QQII", e)
            scratch = self.u("QQ", e + 24)
            out.append((self.heap_name(seg, off), oh, cache, scratch))

    def root(self):
        msgs = self.messages(self.root_oh)
        d = next(d for t, _, d in msgs if t == 0x0011)
        bt, hp = struct.unpack_from("<QQ", d)
        if self.root_scratch is not None:
            assert (bt, hp) == tuple(self.root_scratch), "root scratch-pad = symbol-table message"
        return self.group(bt, hp)


def read(path):
    """The file's content as nested dicts of Dataset objects."""
    return H5Read(path).root()
