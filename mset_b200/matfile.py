"""Reader for MATLAB v7.3 MAT-files (HDF5 containers), written for the
reference's example dataset (examples/CuAu_24size_dataset: 4D-STEM patterns
per tilt, the STEM_data info struct and the stored reconstruction).

No HDF5 library is available, so this module reads the HDF5 structures that
MATLAB writes directly, following the published HDF5 file-format
specification:

* superblock version 0 after MATLAB's 512-byte user block (all addresses are
  relative to the superblock);
* version-1 object headers with continuation blocks;
* groups as symbol tables (version-1 B-tree of group nodes + local heap);
* datasets with compact, contiguous or chunked storage (version-1 B-tree of
  chunks), the deflate and shuffle filters;
* datatypes: integers, IEEE floats, MATLAB's {real, imag} compound for
  complex data, object references (cell arrays);
* the MATLAB_class / MATLAB_empty attributes.

Arrays come back in MATLAB orientation (HDF5 stores MATLAB's column-major
array with the dimensions reversed; the reader transposes).  A struct is a
dict, a cell array a numpy object array, a char array a str.
"""
from __future__ import annotations

import struct
import zlib

import numpy as np

_SIG = b"\x89HDF\r\n\x1a\n"


class MatFileError(ValueError):
    pass


class _File:
    def __init__(self, path: str):
        with open(path, "rb") as f:
            self.buf = f.read()
        base = -1
        for off in (0, 512, 1024, 2048, 4096):
            if self.buf[off:off + 8] == _SIG:
                base = off
                break
        if base < 0:
            raise MatFileError(f"{path}: not an HDF5-based MAT-file (v7.3)")
        self.base = base
        b = self.buf
        ver = b[base + 8]
        if ver not in (0, 1):
            raise MatFileError(f"superblock version {ver} not supported")
        self.so, self.sl = b[base + 13], b[base + 14]
        if self.so != 8 or self.sl != 8:
            raise MatFileError("only 8-byte offsets and lengths are supported")
        p = base + 24 + (4 if ver == 1 else 0)
        # base address, free-space info, end of file, driver info
        p += 32
        self.root = self._symbol_entry(p)[1]

    # -- primitives -------------------------------------------------------------
    def u(self, pos: int, n: int) -> int:
        return int.from_bytes(self.buf[pos:pos + n], "little")

    def addr(self, a: int) -> int:
        return self.base + a

    def _symbol_entry(self, p: int):
        return self.u(p, 8), self.u(p + 8, 8)  # (link name offset, object header address)

    # -- object headers ---------------------------------------------------------
    def messages(self, oh: int):
        """(type, body offset, size) of every message of the object header"""
        p = self.addr(oh)
        if self.buf[p:p + 4] == b"OHDR":
            raise MatFileError("version-2 object headers are not supported")
        if self.buf[p] != 1:
            raise MatFileError(f"object header version {self.buf[p]} not supported")
        nmsg = self.u(p + 2, 2)
        size = self.u(p + 8, 4)
        blocks = [(p + 16, size)]
        out = []
        while blocks and len(out) < nmsg:
            start, length = blocks.pop(0)
            q, end = start, start + length
            while q + 8 <= end and len(out) < nmsg:
                mtype, msize = self.u(q, 2), self.u(q + 2, 2)
                body = q + 8
                if mtype == 0x10:  # continuation
                    blocks.append((self.addr(self.u(body, 8)), self.u(body + 8, 8)))
                out.append((mtype, body, msize))
                q = body + msize
        return out

    # -- groups -----------------------------------------------------------------
    def group_members(self, oh: int) -> dict:
        for mtype, body, _ in self.messages(oh):
            if mtype == 0x11:  # symbol table
                btree, heap = self.u(body, 8), self.u(body + 8, 8)
                hp = self.addr(heap)
                if self.buf[hp:hp + 4] != b"HEAP":
                    raise MatFileError("bad local heap")
                data = self.addr(self.u(hp + 24, 8))
                out = {}
                self._walk_group_tree(btree, data, out)
                return out
        raise MatFileError("object is not a group")

    def _name(self, heap_data: int, off: int) -> str:
        p = heap_data + off
        e = self.buf.index(b"\0", p)
        return self.buf[p:e].decode()

    def _walk_group_tree(self, node: int, heap_data: int, out: dict):
        p = self.addr(node)
        if self.buf[p:p + 4] != b"TREE" or self.buf[p + 4] != 0:
            raise MatFileError("bad group B-tree node")
        level, used = self.buf[p + 5], self.u(p + 6, 2)
        q = p + 24 + 8  # header, then key 0
        for _ in range(used):
            child = self.u(q, 8)
            q += 16  # child, next key
            if level > 0:
                self._walk_group_tree(child, heap_data, out)
                continue
            s = self.addr(child)
            if self.buf[s:s + 4] != b"SNOD":
                raise MatFileError("bad symbol table node")
            for k in range(self.u(s + 6, 2)):
                name_off, ohdr = self._symbol_entry(s + 8 + 40 * k)
                out[self._name(heap_data, name_off)] = ohdr

    # -- datatypes --------------------------------------------------------------
    def datatype(self, p: int):
        """(kind, numpy dtype or member list, size) of a datatype message at p"""
        cls, ver = self.buf[p] & 0x0F, self.buf[p] >> 4
        bits = self.u(p + 1, 3)
        size = self.u(p + 4, 4)
        if cls == 0:
            signed = bool(bits & 0x08)
            order = ">" if bits & 1 else "<"
            return "num", np.dtype(f"{order}{'i' if signed else 'u'}{size}"), size
        if cls == 1:
            order = ">" if bits & 1 else "<"
            return "num", np.dtype(f"{order}f{size}"), size
        if cls == 7:
            return "ref", np.dtype("<u8"), size
        if cls == 3:
            return "str", np.dtype(f"S{size}"), size
        if cls == 9:  # variable length (MATLAB_fields); data in the global heap, not read
            return "vlen", None, size
        if cls == 6:
            nmem = bits & 0xFFFF
            q = p + 8
            members = []
            for _ in range(nmem):
                e = self.buf.index(b"\0", q)
                name = self.buf[q:e].decode()
                if ver < 3:
                    q += (e - q + 8) // 8 * 8
                    off = self.u(q, 4)
                    q += 4 + 28 if ver == 1 else 4
                else:
                    q = e + 1
                    nb = max(1, (size.bit_length() + 7) // 8)
                    off = self.u(q, nb)
                    q += nb
                kind, dt, msz = self.datatype(q)
                q += self._datatype_len(q)
                members.append((name, off, dt))
            return "compound", members, size
        raise MatFileError(f"datatype class {cls} not supported")

    def _datatype_len(self, p: int) -> int:
        cls, ver = self.buf[p] & 0x0F, self.buf[p] >> 4
        if cls in (0,):
            return 12
        if cls == 1:
            return 20
        if cls in (3, 7):
            return 8
        if cls == 9:
            return 8 + self._datatype_len(p + 8)
        if cls == 6:
            bits = self.u(p + 1, 3)
            size = self.u(p + 4, 4)
            q = p + 8
            for _ in range(bits & 0xFFFF):
                e = self.buf.index(b"\0", q)
                if ver < 3:
                    q += (e - q + 8) // 8 * 8
                    q += 4 + 28 if ver == 1 else 4
                else:
                    q = e + 1 + max(1, (size.bit_length() + 7) // 8)
                q += self._datatype_len(q)
            return q - p
        raise MatFileError(f"datatype class {cls} not supported")

    # -- datasets -----------------------------------------------------------------
    def object_info(self, oh: int) -> dict:
        info = {"attrs": {}, "filters": []}
        for mtype, body, msize in self.messages(oh):
            if mtype == 0x01:
                ver, nd, flags = self.buf[body], self.buf[body + 1], self.buf[body + 2]
                q = body + (8 if ver == 1 else 4)
                info["shape"] = tuple(self.u(q + 8 * i, 8) for i in range(nd))
            elif mtype == 0x03:
                info["type"] = self.datatype(body)
            elif mtype == 0x08:
                info["layout"] = self._layout(body)
            elif mtype == 0x0B:
                info["filters"] = self._filters(body)
            elif mtype == 0x0C:
                name, val = self._attribute(body)
                info["attrs"][name] = val
            elif mtype == 0x11:
                info["group"] = True
        return info

    def _layout(self, p: int):
        ver = self.buf[p]
        if ver != 3:
            raise MatFileError(f"data layout version {ver} not supported")
        cls = self.buf[p + 1]
        if cls == 0:
            n = self.u(p + 2, 2)
            return ("compact", p + 4, n)
        if cls == 1:
            return ("contiguous", self.u(p + 2, 8), self.u(p + 10, 8))
        if cls == 2:
            nd = self.buf[p + 2]
            btree = self.u(p + 3, 8)
            dims = [self.u(p + 11 + 4 * i, 4) for i in range(nd)]
            return ("chunked", btree, dims)
        raise MatFileError(f"layout class {cls} not supported")

    def _filters(self, p: int):
        ver, n = self.buf[p], self.buf[p + 1]
        q = p + (8 if ver == 1 else 2)
        out = []
        for _ in range(n):
            fid = self.u(q, 2)
            if ver == 1:
                namelen, nvals = self.u(q + 2, 2), self.u(q + 6, 2)
                q += 8 + (namelen + 7) // 8 * 8
            elif fid >= 256:
                namelen, nvals = self.u(q + 2, 2), self.u(q + 6, 2)
                q += 8 + namelen
            else:
                nvals = self.u(q + 4, 2)
                q += 6
            vals = [self.u(q + 4 * i, 4) for i in range(nvals)]
            q += 4 * nvals
            if ver == 1 and nvals % 2:
                q += 4
            out.append((fid, vals))
        return out

    def _attribute(self, p: int):
        ver = self.buf[p]
        nlen, tlen, slen = self.u(p + 2, 2), self.u(p + 4, 2), self.u(p + 6, 2)
        if ver == 1:
            q = p + 8
            name = self.buf[q:q + nlen].split(b"\0")[0].decode()
            q += (nlen + 7) // 8 * 8
            tp = q
            q += (tlen + 7) // 8 * 8
            sp = q
            q += (slen + 7) // 8 * 8
        else:
            q = p + 8 + (1 if ver == 3 else 0)
            name = self.buf[q:q + nlen].split(b"\0")[0].decode()
            q += nlen
            tp = q
            q += tlen
            sp = q
            q += slen
        kind, dt, size = self.datatype(tp)
        sver, nd = self.buf[sp], self.buf[sp + 1]
        dq = sp + (8 if sver == 1 else 4)
        shape = tuple(self.u(dq + 8 * i, 8) for i in range(nd))
        count = int(np.prod(shape)) if shape else 1
        raw = self.buf[q:q + count * size]
        if kind == "str":
            return name, raw.split(b"\0")[0].decode(errors="replace")
        if kind == "num":
            return name, np.frombuffer(raw, dt, count).reshape(shape) if shape else np.frombuffer(raw, dt, 1)[0]
        return name, None

    def _raw(self, info: dict) -> bytes:
        shape = info["shape"]
        kind, dt, size = info["type"]
        count = int(np.prod(shape)) if shape else 1
        lay = info["layout"]
        if lay[0] == "compact":
            return self.buf[lay[1]:lay[1] + lay[2]]
        if lay[0] == "contiguous":
            if lay[1] == (1 << 64) - 1:
                return bytes(count * size)
            a = self.addr(lay[1])
            return self.buf[a:a + count * size]
        # chunked: assemble the chunks into a C-order array of the full shape
        cdims = lay[2][:-1]
        out = np.zeros(tuple(shape), dtype=np.dtype(f"V{size}"))
        self._walk_chunks(lay[1], len(shape), cdims, info["filters"], size, out)
        return out.tobytes()

    def _walk_chunks(self, node, rank, cdims, filters, esize, out):
        p = self.addr(node)
        if self.buf[p:p + 4] != b"TREE" or self.buf[p + 4] != 1:
            raise MatFileError("bad chunk B-tree node")
        level, used = self.buf[p + 5], self.u(p + 6, 2)
        ksize = 8 + 8 * (rank + 1)
        q = p + 24
        for _ in range(used):
            csize, mask = self.u(q, 4), self.u(q + 4, 4)
            offs = [self.u(q + 8 + 8 * i, 8) for i in range(rank)]
            child = self.u(q + ksize, 8)
            q += ksize + 8
            if level > 0:
                self._walk_chunks(child, rank, cdims, filters, esize, out)
                continue
            a = self.addr(child)
            data = self.buf[a:a + csize]
            for i, (fid, vals) in enumerate(reversed(filters)):
                if mask & (1 << (len(filters) - 1 - i)):
                    continue
                if fid == 1:
                    data = zlib.decompress(data)
                elif fid == 2:
                    n = len(data) // esize
                    data = np.frombuffer(data, np.uint8).reshape(esize, n).T.tobytes()
                else:
                    raise MatFileError(f"filter {fid} not supported")
            chunk = np.frombuffer(data, dtype=out.dtype, count=int(np.prod(cdims))).reshape(cdims)
            sl = tuple(slice(o, min(o + c, s)) for o, c, s in zip(offs, cdims, out.shape))
            out[sl] = chunk[tuple(slice(0, x.stop - x.start) for x in sl)]

    # -- MATLAB values ------------------------------------------------------------
    def value(self, oh: int):
        info = self.object_info(oh)
        if info.get("group"):
            members = self.group_members(oh)
            return {k: self.value(v) for k, v in members.items() if not k.startswith("#")}
        mclass = info["attrs"].get("MATLAB_class", "")
        shape = info["shape"]
        if "MATLAB_empty" in info["attrs"] and np.any(info["attrs"]["MATLAB_empty"]):
            return np.zeros((0, 0))
        kind, dt, size = info["type"]
        raw = self._raw(info)
        count = int(np.prod(shape)) if shape else 1
        if kind == "compound":
            names = {m[0]: m for m in dt}
            rec = np.dtype({"names": [m[0] for m in dt], "formats": [m[2] for m in dt],
                            "offsets": [m[1] for m in dt], "itemsize": size})
            a = np.frombuffer(raw, rec, count).reshape(shape)
            if "real" in names and "imag" in names:
                arr = a["real"] + 1j * a["imag"]
            else:
                return a
        elif kind == "ref":
            refs = np.frombuffer(raw, "<u8", count).reshape(shape)
            cells = np.empty(shape, dtype=object)
            for idx in np.ndindex(*shape):
                cells[idx] = self.value(int(refs[idx]))
            return cells.T
        else:
            arr = np.frombuffer(raw, dt, count).reshape(shape)
        if mclass == "char":
            return "".join(chr(c) for c in arr.T.reshape(-1, order="F"))
        if mclass == "logical":
            arr = arr.astype(bool)
        return np.ascontiguousarray(arr.T)


def loadmat73(path: str, names=None) -> dict:
    """{variable name: value} of a v7.3 MAT-file (all variables, or `names`)"""
    f = _File(path)
    top = f.group_members(f.root)
    out = {}
    for k, oh in top.items():
        if k.startswith("#") or (names is not None and k not in names):
            continue
        out[k] = f.value(oh)
    return out
