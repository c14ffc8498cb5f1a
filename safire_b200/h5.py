"""Read-only HDF5 reader for the files the reference's AFQMC executable reads and writes.

No libhdf5 / h5py is assumed: this module parses the subset of the HDF5 on-disk format (the
public "HDF5 File Format Specification", versions 0-1 superblocks) that these files use —
symbol-table groups (v1 B-tree of SNOD nodes over a local heap), version-1 object headers with
continuation blocks, dataspaces v1/v2, contiguous / compact / chunked (v1 B-tree, deflate and
shuffle filters) layouts, fixed-point, floating-point, fixed and variable-length string,
compound, enum and array datatypes, and attributes.  Complex numbers stored as a compound
{r, i} of two floats come back as numpy complex arrays.

The Hamiltonian reader (RealDenseHamiltonian.cpp:74-134, hdf5_helpers.hpp:84-106), the
wavefunction readers (readWfn.cpp:66-200, readWfn.h:88-150) and the sparse-matrix layout
(csr_utils.hpp:344-420) of the reference sit on top of it in safire_b200/inputs.py.

Anything outside that subset (superblock v2/v3, version-2 "OHDR" object headers, new-style
link-message groups, dense attribute storage, other filters) raises H5Unsupported.
"""
from __future__ import annotations

import zlib

import numpy as np


class H5Unsupported(NotImplementedError):
    pass


_SIG = b"\x89HDF\r\n\x1a\n"
_UNDEF = 0xFFFFFFFFFFFFFFFF


class _VLenString:
    """Marker dtype: variable-length string stored in a global heap."""


class _Type:
    """A parsed datatype: numpy dtype (or _VLenString) and the byte size of one element."""

    def __init__(self, dtype, size, complex_pair=False):
        self.dtype, self.size, self.complex_pair = dtype, size, complex_pair


class File:
    """An HDF5 file opened for reading: `f["Hamiltonian/hcore"]` reads a dataset into numpy,
    `f.attrs(path)` the attributes of a group or dataset, `f.keys(path)` a group's members."""

    def __init__(self, path):
        with open(path, "rb") as fh:
            self.buf = fh.read()
        b = self.buf
        # the superblock sits at byte 0 or at a power of two from 512 on (a user block before it)
        sb = next((o for o in [0] + [512 << k for k in range(24)]
                   if o < len(b) and b[o:o + 8] == _SIG), -1)
        if sb < 0:
            raise ValueError(f"{path}: not an HDF5 file")
        ver = b[sb + 8]
        if ver not in (0, 1):
            raise H5Unsupported(f"superblock version {ver}")
        self.O, self.L = b[sb + 13], b[sb + 14]
        p = sb + 24 + (4 if ver == 1 else 0)
        self.base = self._u(p, self.O)
        p += 4 * self.O  # base, free-space, end-of-file, driver-info addresses
        self.root = self._entry(p)[1]
        self._gheap = {}

    # ---------------------------------------------------------------- primitives
    def _u(self, p, n):
        return int.from_bytes(self.buf[p:p + n], "little")

    def _a(self, addr):
        return self.base + addr

    def _entry(self, p):
        """Symbol table entry: (link name heap offset, object header address, cache type,
        scratch bytes)."""
        name_off = self._u(p, self.O)
        hdr = self._u(p + self.O, self.O)
        cache = self._u(p + 2 * self.O, 4)
        return name_off, hdr, cache, self.buf[p + 2 * self.O + 8:p + 2 * self.O + 24]

    def _cstr(self, p):
        e = self.buf.index(b"\0", p)
        return self.buf[p:e].decode()

    # ---------------------------------------------------------------- object headers
    def _messages(self, addr):
        """[(type, flags, data offset, size)] of a version-1 object header."""
        p = self._a(addr)
        b = self.buf
        if b[p:p + 4] == b"OHDR":
            raise H5Unsupported("version-2 object headers")
        if b[p] != 1:
            raise H5Unsupported(f"object header version {b[p]}")
        nmsg = self._u(p + 2, 2)
        size = self._u(p + 8, 4)
        blocks = [(p + 16, size)]
        out = []
        while blocks and len(out) < nmsg:
            q, n = blocks.pop(0)
            end = q + n
            while q + 8 <= end and len(out) < nmsg:
                mtype, msize, mflags = self._u(q, 2), self._u(q + 2, 2), b[q + 4]
                d = q + 8
                if mtype == 0x10:  # continuation
                    blocks.append((self._a(self._u(d, self.O)), self._u(d + self.O, self.L)))
                out.append((mtype, mflags, d, msize))
                q = d + msize
        return out

    # ---------------------------------------------------------------- groups
    def _group_members(self, addr):
        """{name: object header address} of a symbol-table group."""
        btree = heap = None
        for mtype, _, d, _ in self._messages(addr):
            if mtype == 0x11:
                btree, heap = self._u(d, self.O), self._u(d + self.O, self.O)
            elif mtype in (0x06, 0x02):
                raise H5Unsupported("new-style (link message) groups")
        if btree is None:
            raise KeyError("not a group")
        hp = self._a(heap)
        if self.buf[hp:hp + 4] != b"HEAP":
            raise ValueError("bad local heap")
        data = self._a(self._u(hp + 8 + 2 * self.L, self.O))
        out = {}
        self._walk_group_tree(btree, data, out)
        return out

    def _walk_group_tree(self, addr, heap_data, out):
        p = self._a(addr)
        b = self.buf
        if b[p:p + 4] != b"TREE" or b[p + 4] != 0:
            raise ValueError("bad group B-tree node")
        level, used = b[p + 5], self._u(p + 6, 2)
        q = p + 8 + 2 * self.O + self.L  # past siblings and key 0
        for _ in range(used):
            child = self._u(q, self.O)
            q += self.O + self.L
            if level > 0:
                self._walk_group_tree(child, heap_data, out)
                continue
            s = self._a(child)
            if b[s:s + 4] != b"SNOD":
                raise ValueError("bad symbol table node")
            nsym = self._u(s + 6, 2)
            e = s + 8
            for _ in range(nsym):
                name_off, hdr, _, _ = self._entry(e)
                out[self._cstr(heap_data + name_off)] = hdr
                e += 2 * self.O + 24

    def _resolve(self, path):
        addr = self.root
        for part in [x for x in path.strip("/").split("/") if x]:
            members = self._group_members(addr)
            if part not in members:
                raise KeyError(path)
            addr = members[part]
        return addr

    def keys(self, path="/"):
        return sorted(self._group_members(self._resolve(path)))

    def is_group(self, path):
        try:
            return any(m[0] == 0x11 for m in self._messages(self._resolve(path)))
        except KeyError:
            return False

    def __contains__(self, path):
        try:
            self._resolve(path)
            return True
        except KeyError:
            return False

    # ---------------------------------------------------------------- datatypes / dataspaces
    def _dtype(self, p):
        """(_Type, bytes consumed) of the datatype message at p."""
        b = self.buf
        cls, ver = b[p] & 0x0F, b[p] >> 4
        bits = self._u(p + 1, 3)
        size = self._u(p + 4, 4)
        q = p + 8
        order = ">" if bits & 1 else "<"
        if cls == 0:  # fixed point
            kind = "i" if bits & 0x08 else "u"
            return _Type(np.dtype(f"{order}{kind}{size}"), size), 8 + 4
        if cls == 1:  # floating point
            return _Type(np.dtype(f"{order}f{size}"), size), 8 + 12
        if cls == 3:  # fixed-length string
            return _Type(np.dtype(f"S{size}"), size), 8
        if cls == 4:  # bitfield
            return _Type(np.dtype(f"{order}u{size}"), size), 8 + 4
        if cls == 6:  # compound
            nmem = bits & 0xFFFF
            names, formats, offsets = [], [], []
            for _ in range(nmem):
                name = self._cstr(q)
                n = len(name) + 1
                if ver < 3:
                    q += (n + 7) // 8 * 8
                    off = self._u(q, 4)
                    q += 4
                    if ver == 1:
                        q += 1 + 3 + 4 + 4 + 16  # rank, reserved, permutation, reserved, dims
                else:
                    q += n
                    nb = 1 if size < 256 else 2 if size < 65536 else 3 if size < (1 << 24) else 4
                    off = self._u(q, nb)
                    q += nb
                t, used = self._dtype(q)
                q += used
                names.append(name)
                formats.append(t.dtype if not isinstance(t.dtype, type) else np.dtype("O"))
                offsets.append(off)
            dt = np.dtype({"names": names, "formats": formats, "offsets": offsets,
                           "itemsize": size})
            pair = (nmem == 2 and all(f.kind == "f" and f == formats[0] for f in formats)
                    and offsets == [0, formats[0].itemsize])
            return _Type(dt, size, complex_pair=pair), q - p
        if cls == 8:  # enum: base type, then names and values
            base, used = self._dtype(q)
            q += used
            nmem = bits & 0xFFFF
            for _ in range(nmem):
                n = len(self._cstr(q)) + 1
                q += n if ver >= 3 else (n + 7) // 8 * 8
            q += nmem * base.size
            return _Type(base.dtype, size), q - p
        if cls == 9:  # variable length
            base, used = self._dtype(q)
            if bits & 0x0F == 1:
                return _Type(_VLenString, size), 8 + used
            raise H5Unsupported("variable-length sequences")
        if cls == 10:  # array
            rank = b[q]
            q += 1 if ver >= 3 else 4
            dims = [self._u(q + 4 * i, 4) for i in range(rank)]
            q += 4 * rank + (4 * rank if ver < 3 else 0)
            base, used = self._dtype(q)
            q += used
            return _Type(np.dtype((base.dtype, tuple(dims))), size), q - p
        raise H5Unsupported(f"datatype class {cls}")

    def _dataspace(self, p):
        b = self.buf
        ver, rank, flags = b[p], b[p + 1], b[p + 2]
        if ver == 1:
            q = p + 8
        elif ver == 2:
            if b[p + 3] == 2:  # null dataspace
                return None
            q = p + 4
        else:
            raise H5Unsupported(f"dataspace version {ver}")
        return tuple(self._u(q + self.L * i, self.L) for i in range(rank))

    # ---------------------------------------------------------------- raw data
    def _vlen_strings(self, raw, n):
        out = []
        step = 4 + self.O + 4
        for i in range(n):
            r = raw[i * step:(i + 1) * step]
            ln = int.from_bytes(r[:4], "little")
            coll = int.from_bytes(r[4:4 + self.O], "little")
            idx = int.from_bytes(r[4 + self.O:], "little")
            out.append(self._gheap_object(coll, idx)[:ln].decode(errors="replace"))
        return out

    def _gheap_object(self, coll, idx):
        if coll not in self._gheap:
            p = self._a(coll)
            b = self.buf
            if b[p:p + 4] != b"GCOL":
                raise ValueError("bad global heap collection")
            size = self._u(p + 8, self.L)
            end, q, objs = p + size, p + 8 + self.L, {}
            while q + 8 + self.L <= end:
                oid = self._u(q, 2)
                osz = self._u(q + 8, self.L)
                if oid == 0:
                    break
                d = q + 8 + self.L
                objs[oid] = b[d:d + osz]
                q = d + (osz + 7) // 8 * 8
            self._gheap[coll] = objs
        return self._gheap[coll][idx]

    def _decode(self, raw, t, shape):
        n = int(np.prod(shape)) if shape else 1
        if t.dtype is _VLenString:
            vals = self._vlen_strings(raw, n)
            return vals[0] if shape == () else np.array(vals, dtype=object).reshape(shape)
        a = np.frombuffer(raw, dtype=t.dtype, count=n)
        if t.complex_pair:
            f = t.dtype.fields
            (n0, (d0, _)), (n1, _) = list(f.items())[:2]
            c = np.empty(n, dtype=np.complex128 if d0.itemsize == 8 else np.complex64)
            c.real, c.imag = a[n0], a[n1]
            a = c
        elif a.dtype.kind in "iuf" and a.dtype.byteorder == ">":
            a = a.astype(a.dtype.newbyteorder("="))
        a = a.reshape(shape) if shape else a.reshape(())
        if a.dtype.kind == "S":
            a = np.char.decode(np.char.rstrip(a, b"\0"), errors="replace")
        return a.copy()

    def _chunked(self, btree, rank, chunk, esize, shape, filters):
        if not shape:
            raise H5Unsupported("chunked scalar dataset")
        full = np.zeros(shape, dtype=f"V{esize}")
        self._walk_chunks(btree, rank, chunk, esize, shape, filters, full)
        return full.tobytes()

    def _walk_chunks(self, addr, rank, chunk, esize, shape, filters, full):
        p = self._a(addr)
        b = self.buf
        if b[p:p + 4] != b"TREE" or b[p + 4] != 1:
            raise ValueError("bad chunk B-tree node")
        level, used = b[p + 5], self._u(p + 6, 2)
        q = p + 8 + 2 * self.O
        ksz = 8 + 8 * (rank + 1)
        for _ in range(used):
            csize, mask = self._u(q, 4), self._u(q + 4, 4)
            offs = [self._u(q + 8 + 8 * i, 8) for i in range(rank)]
            child = self._u(q + ksz, self.O)
            q += ksz + self.O
            if level > 0:
                self._walk_chunks(child, rank, chunk, esize, shape, filters, full)
                continue
            raw = b[self._a(child):self._a(child) + csize]
            for i, (fid, _) in reversed(list(enumerate(filters))):
                if mask & (1 << i):
                    continue
                if fid == 1:
                    raw = zlib.decompress(raw)
                elif fid == 2:
                    n = len(raw) // esize
                    raw = np.frombuffer(raw, np.uint8).reshape(esize, n).T.tobytes()
                elif fid == 3:
                    raw = raw[:-4]
                else:
                    raise H5Unsupported(f"filter {fid}")
            blk = np.frombuffer(raw, dtype=f"V{esize}").reshape(chunk)
            sl = tuple(slice(o, min(o + c, s)) for o, c, s in zip(offs, chunk, shape))
            full[sl] = blk[tuple(slice(0, x.stop - x.start) for x in sl)]

    # ---------------------------------------------------------------- datasets / attributes
    def read(self, path):
        msgs = self._messages(self._resolve(path))
        t = shape = layout = None
        filters = []
        for mtype, flags, d, _ in msgs:
            if flags & 0x02:
                raise H5Unsupported("shared header messages")
            if mtype == 0x01:
                shape = self._dataspace(d)
            elif mtype == 0x03:
                t = self._dtype(d)[0]
            elif mtype == 0x08:
                layout = d
            elif mtype == 0x0B:
                filters = self._filters(d)
        if t is None or layout is None:
            raise KeyError(f"{path} is not a dataset")
        shape = shape or ()
        n = int(np.prod(shape)) if shape else 1
        nbytes = n * t.size
        b = self.buf
        ver = b[layout]
        if ver in (1, 2):
            rank, cls = b[layout + 1], b[layout + 2]
            q = layout + 8
            if cls == 0:
                q += 4 * rank
                sz = self._u(q, 4)
                raw = b[q + 4:q + 4 + sz]
            else:
                addr = self._u(q, self.O)
                dims = [self._u(q + self.O + 4 * i, 4) for i in range(rank)]
                if cls == 1:
                    raw = (bytes(nbytes) if addr == _UNDEF
                           else b[self._a(addr):self._a(addr) + nbytes])
                else:
                    raw = self._chunked(addr, rank - 1, dims[:-1], t.size, shape, filters)
        elif ver == 3:
            cls = b[layout + 1]
            q = layout + 2
            if cls == 0:
                sz = self._u(q, 2)
                raw = b[q + 2:q + 2 + sz]
            elif cls == 1:
                addr = self._u(q, self.O)
                raw = bytes(nbytes) if addr == _UNDEF else b[self._a(addr):self._a(addr) + nbytes]
            elif cls == 2:
                rank = b[q]
                addr = self._u(q + 1, self.O)
                dims = [self._u(q + 1 + self.O + 4 * i, 4) for i in range(rank)]
                raw = (bytes(nbytes) if addr == _UNDEF
                       else self._chunked(addr, rank - 1, dims[:-1], t.size, shape, filters))
            else:
                raise H5Unsupported(f"layout class {cls}")
        else:
            raise H5Unsupported(f"data layout version {ver}")
        return self._decode(raw, t, shape)

    __getitem__ = read

    def _filters(self, d):
        b = self.buf
        ver, nf = b[d], b[d + 1]
        q = d + (8 if ver == 1 else 2)
        out = []
        for _ in range(nf):
            fid = self._u(q, 2)
            if ver == 1 or fid >= 256:
                nlen = self._u(q + 2, 2)
                q += 4
            else:
                nlen = 0
                q += 2
            flags, nval = self._u(q, 2), self._u(q + 2, 2)
            q += 4
            q += ((nlen + 7) // 8 * 8) if ver == 1 else nlen
            q += 4 * nval + (4 if ver == 1 and nval % 2 else 0)
            out.append((fid, flags))
        return out

    def attrs(self, path="/"):
        """{name: value} of the attributes of the object at path."""
        out = {}
        b = self.buf
        for mtype, _, d, _ in self._messages(self._resolve(path)):
            if mtype == 0x15:
                raise H5Unsupported("dense attribute storage")
            if mtype != 0x0C:
                continue
            ver = b[d]
            nlen, tlen, slen = self._u(d + 2, 2), self._u(d + 4, 2), self._u(d + 6, 2)
            if ver == 1:
                pad = lambda x: (x + 7) // 8 * 8  # noqa: E731
                q = d + 8
                name = self._cstr(q)
                q += pad(nlen)
                t = self._dtype(q)[0]
                q += pad(tlen)
                shape = self._dataspace(q)
                q += pad(slen)
            else:
                q = d + 8 + (1 if ver == 3 else 0)
                name = self._cstr(q)
                q += nlen
                t = self._dtype(q)[0]
                q += tlen
                shape = self._dataspace(q)
                q += slen
            shape = shape or ()
            n = int(np.prod(shape)) if shape else 1
            step = (4 + self.O + 4) if t.dtype is _VLenString else t.size
            v = self._decode(b[q:q + n * step], t, shape)
            out[name] = v.item() if isinstance(v, np.ndarray) and v.shape == () else v
        return out

    def walk(self, path="/"):
        """Every dataset path below `path` (depth first)."""
        out = []
        for k in self.keys(path):
            sub = path.rstrip("/") + "/" + k
            if self.is_group(sub):
                out += self.walk(sub)
            else:
                out.append(sub)
        return out
