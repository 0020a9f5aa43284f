"""Structural reader for the HDF5 map files the library writes (test helper).

Walks the classic-format objects such a file holds (superblock v0, symbol
table root group, version-1 object headers) and returns, per dataset, its
dataspace, element size, raw data address and attributes.  Attribute values
are decoded for the types the map files use: fixed strings, variable-length
sequences of object references and variable-length strings (resolved through
the global heap) and the {object reference, int32} compound of
REFERENCE_LIST.  Used only to check the writer's output.
"""
import struct


class H5Struct:
    def __init__(self, path):
        self.b = open(path, "rb").read()
        b = self.b
        assert b[:8] == b"\x89HDF\r\n\x1a\n", "not an HDF5 file"
        assert b[8] == 0, "superblock version"
        assert b[13] == 8 and b[14] == 8
        self.leaf_k, self.int_k = self.u(16, 2), self.u(18, 2)
        self.eof = self.u(40, 8)
        re = 56
        assert self.u(re + 16, 4) == 1
        self.btree, self.heap = self.u(re + 24, 8), self.u(re + 32, 8)
        self.root_oh = self.u(re + 8, 8)
        assert b[self.heap:self.heap + 4] == b"HEAP"
        self.heap_size = self.u(self.heap + 8, 8)
        self.heap_free = self.u(self.heap + 16, 8)
        self.heap_data = self.u(self.heap + 24, 8)
        self.objects = {}  # name -> object header address
        self.keys = []
        self._walk(self.btree)

    def u(self, off, n):
        return int.from_bytes(self.b[off:off + n], "little")

    def name_at(self, off):
        p = self.heap_data + off
        return self.b[p:self.b.index(0, p)].decode()

    def _walk(self, node):
        b = self.b
        assert b[node:node + 4] == b"TREE" and b[node + 4] == 0
        level, used = b[node + 5], self.u(node + 6, 2)
        p = node + 24
        keys = [self.u(p, 8)]
        p += 8
        for _ in range(used):
            child = self.u(p, 8)
            keys.append(self.u(p + 8, 8))
            p += 16
            if level > 0:
                self._walk(child)
                continue
            assert b[child:child + 4] == b"SNOD"
            n = self.u(child + 6, 2)
            e = child + 8
            for _ in range(n):
                self.objects[self.name_at(self.u(e, 8))] = self.u(e + 8, 8)
                e += 40
        self.keys = keys

    def messages(self, addr, strict=False):
        """Messages of the object header at addr, following continuation
        blocks.  strict: a single block that its messages fill exactly (the
        layout the writer produces)."""
        b = self.b
        assert b[addr] == 1, "object header version"
        nmsg, hsize = self.u(addr + 2, 2), self.u(addr + 8, 4)
        out, blocks, i = [], [(addr + 16, hsize)], 0
        while i < len(blocks):
            p, end = blocks[i][0], blocks[i][0] + blocks[i][1]
            i += 1
            while p + 8 <= end and len(out) < nmsg:
                t, sz, fl = self.u(p, 2), self.u(p + 2, 2), b[p + 4]
                out.append((t, fl, b[p + 8:p + 8 + sz]))
                if t == 0x10:
                    blocks.append((self.u(p + 8, 8), self.u(p + 16, 8)))
                p += 8 + sz
            if strict:
                assert len(blocks) == 1 and p == end, "messages must fill the header exactly"
        assert len(out) == nmsg
        return out

    def gheap(self, addr, idx):
        b = self.b
        assert b[addr:addr + 4] == b"GCOL"
        size = self.u(addr + 8, 8)
        p = addr + 16
        while p < addr + size:
            i, sz = self.u(p, 2), self.u(p + 8, 8)
            if i == idx:
                return b[p + 16:p + 16 + sz]
            if i == 0:
                break
            p += 16 + (sz + 7) // 8 * 8
        raise KeyError(idx)

    def dataset(self, name, strict=False):
        d = dict(attrs={})
        for t, fl, body in self.messages(self.objects[name], strict):
            if t == 0x1:
                rank = body[1]
                d["dims"] = [struct.unpack_from("<Q", body, 8 + 8 * i)[0] for i in range(rank)]
            elif t == 0x3:
                d["class"], d["elsize"] = body[0] & 0xF, struct.unpack_from("<I", body, 4)[0]
            elif t == 0x8:
                assert body[0] == 3 and body[1] == 1
                d["addr"], d["size"] = struct.unpack_from("<QQ", body, 2)
            elif t == 0xC:
                nl, dl, sl = struct.unpack_from("<HHH", body, 2)
                pad = lambda n: (n + 7) // 8 * 8
                an = body[8:8 + nl - 1].decode()
                dt = body[8 + pad(nl):8 + pad(nl) + dl]
                ds = body[8 + pad(nl) + pad(dl):8 + pad(nl) + pad(dl) + sl]
                data = body[8 + pad(nl) + pad(dl) + pad(sl):]
                d["attrs"][an] = self._attr_value(dt, ds, data)
        return d

    def _attr_value(self, dt, ds, data):
        cls = dt[0] & 0xF
        rank = ds[1]
        n = 1
        for i in range(rank):
            n *= struct.unpack_from("<Q", ds, 8 + 8 * i)[0]
        if cls == 3:  # fixed string
            size = struct.unpack_from("<I", dt, 4)[0]
            return data[:size].split(b"\0")[0].decode()
        if cls == 9:  # variable length: resolve each element in the global heap
            vals = []
            for e in range(n):
                ln, addr, idx = struct.unpack_from("<IQI", data, 16 * e)
                obj = self.gheap(addr, idx)
                if dt[1] & 0xF == 1:
                    vals.append(obj[:ln].decode())
                else:
                    vals.append([struct.unpack_from("<Q", obj, 8 * q)[0] for q in range(ln)])
            return vals
        if cls == 6:  # REFERENCE_LIST compound
            return [struct.unpack_from("<Qi", data, 16 * e) for e in range(n)]
        return data
