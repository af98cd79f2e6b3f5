"""A small read-only HDF5 reader for the reference's Hamiltonian, wavefunction and results files.

Written from the published HDF5 file format specification (version 0 superblock, version 1
object headers, symbol-table groups); it reads what those files use and rejects the rest loudly:

  * superblock versions 0 and 1, 8-byte offsets and lengths;
  * groups as symbol tables (version 1 B-tree of type 0 + local heap + SNOD nodes), link messages
    of version 2 object headers are not read;
  * datasets with compact, contiguous or chunked layout (version 1 B-tree of type 1; the deflate
    and shuffle filters);
  * datatypes: fixed point, floating point, fixed-length strings, enums (h5py's bool), compounds
    (h5py's complex numbers {r, i}), variable-length strings (global heap);
  * attributes (message 0x000C, versions 1-3).

    f = H5File(path)
    f["Hamiltonian/hcore"]                 # numpy array (complex compounds become complex128)
    f.attrs("Hamiltonian")["nuclear_energy"]
    f.keys("Hamiltonian")

The readers of the reference this serves: RealDenseHamiltonian.cpp:77-134 (hcore, DenseFactorized/L,
read_energy_offset in hdf5_helpers.hpp:84-106), readWfn.cpp:50-131 and csr_utils.hpp:345-420
(Wavefunction/NOMSD, PsiT_n in CSR), and the results files the functional tests write.
"""
import struct
import zlib

import numpy as np

_SIG = b"\x89HDF\r\n\x1a\n"
_UNDEF = 0xFFFFFFFFFFFFFFFF


class H5Error(ValueError):
    pass


class _Type:
    """A parsed datatype: numpy dtype for fixed-size data, or a marker for variable-length strings."""

    def __init__(self, cls, size, dtype=None, vlen_str=False, enum=None, base=None):
        self.cls, self.size, self.dtype, self.vlen_str, self.enum, self.base = cls, size, dtype, vlen_str, enum, base


class H5File:
    def __init__(self, path):
        with open(path, "rb") as fh:
            self.b = fh.read()
        self.path = path
        b = self.b
        if b[:8] != _SIG:
            raise H5Error(f"{path}: not an HDF5 file (signature at offset 0 only)")
        ver = b[8]
        if ver not in (0, 1):
            raise H5Error(f"{path}: superblock version {ver} not supported")
        self.so, self.sl = b[13], b[14]
        if self.so != 8 or self.sl != 8:
            raise H5Error(f"{path}: offset/length sizes {self.so}/{self.sl} not supported")
        p = 24 + (4 if ver == 1 else 0)
        self.base = self._u(p, 8)
        p += 32  # base, free-space, end of file, driver info addresses
        # root group symbol table entry
        self.root = self._entry(p)

    # -- primitives -----------------------------------------------------------------------------
    def _u(self, p, n):
        return int.from_bytes(self.b[p:p + n], "little")

    def _entry(self, p):
        """Symbol table entry: (name offset, object header address, cache type, B-tree, heap)."""
        name_off, hdr = self._u(p, 8), self._u(p + 8, 8)
        cache = self._u(p + 16, 4)
        btree = heap = None
        if cache == 1:
            btree, heap = self._u(p + 24, 8), self._u(p + 32, 8)
        return dict(name_off=name_off, hdr=hdr, cache=cache, btree=btree, heap=heap)

    def _heap_data(self, addr):
        b = self.b
        if b[addr:addr + 4] != b"HEAP":
            raise H5Error(f"local heap signature missing at {addr}")
        return self._u(addr + 24, 8)

    def _cstr(self, p):
        e = self.b.index(b"\0", p)
        return self.b[p:e].decode()

    # -- object headers -------------------------------------------------------------------------
    def _messages(self, addr):
        b = self.b
        if b[addr:addr + 4] == b"OHDR":
            raise H5Error("version 2 object headers are not supported")
        if b[addr] != 1:
            raise H5Error(f"object header version {b[addr]} at {addr}")
        nmsg = self._u(addr + 2, 2)
        size = self._u(addr + 8, 4)
        blocks = [(addr + 16, size)]
        out = []
        while blocks and len(out) < nmsg:
            start, length = blocks.pop(0)
            p, end = start, start + length
            while p + 8 <= end and len(out) < nmsg:
                mtype, msize, flags = self._u(p, 2), self._u(p + 2, 2), b[p + 4]
                data = p + 8
                if mtype == 0x10:  # continuation
                    blocks.append((self._u(data, 8), self._u(data + 8, 8)))
                out.append((mtype, data, msize, flags))
                p = data + msize
        return out

    # -- datatypes and dataspaces ---------------------------------------------------------------
    def _dtype(self, p):
        b = self.b
        cls, ver = b[p] & 0x0F, b[p] >> 4
        bf = b[p + 1] | (b[p + 2] << 8) | (b[p + 3] << 16)
        size = self._u(p + 4, 4)
        q = p + 8
        if cls == 0:  # fixed point
            order = ">" if bf & 1 else "<"
            signed = bool(bf & 8)
            return _Type(0, size, np.dtype(f"{order}{'i' if signed else 'u'}{size}")), q + 4
        if cls == 1:  # floating point
            order = ">" if bf & 1 else "<"
            if size not in (2, 4, 8):
                raise H5Error(f"float of {size} bytes")
            return _Type(1, size, np.dtype(f"{order}f{size}")), q + 12
        if cls == 3:  # fixed-length string
            return _Type(3, size, np.dtype(f"S{size}")), q
        if cls == 6:  # compound
            nmem = bf & 0xFFFF
            names, formats, offsets = [], [], []
            for _ in range(nmem):
                name = self._cstr(q)
                if ver < 3:
                    q += (len(name) + 8) // 8 * 8
                else:
                    q += len(name) + 1
                if ver == 1:
                    off = self._u(q, 4)
                    q += 4 + 1 + 3 + 4 + 4 + 16
                elif ver == 2:
                    off = self._u(q, 4)
                    q += 4
                else:
                    nb = max(1, (size.bit_length() + 7) // 8)
                    off = self._u(q, nb)
                    q += nb
                t, q = self._dtype(q)
                if t.dtype is None:
                    raise H5Error("compound member without a fixed-size type")
                names.append(name)
                formats.append(t.dtype)
                offsets.append(off)
            return _Type(6, size, np.dtype(dict(names=names, formats=formats, offsets=offsets, itemsize=size))), q
        if cls == 8:  # enum: base type, names, values
            base, q = self._dtype(q)
            nmem = bf & 0xFFFF
            names = []
            for _ in range(nmem):
                name = self._cstr(q)
                names.append(name)
                q += (len(name) + 8) // 8 * 8 if ver < 3 else len(name) + 1
            vals = np.frombuffer(self.b, base.dtype, nmem, q)
            q += nmem * base.size
            return _Type(8, size, base.dtype, enum=dict(zip(vals.tolist(), names))), q
        if cls == 9:  # variable length
            kind = bf & 0xF
            base, q = self._dtype(q)
            if kind == 1:
                return _Type(9, size, None, vlen_str=True), q
            raise H5Error("variable-length sequences are not supported")
        raise H5Error(f"datatype class {cls} not supported")

    def _space(self, p):
        b = self.b
        ver, rank = b[p], b[p + 1]
        if ver == 1:
            q = p + 8
        elif ver == 2:
            if b[p + 3] == 0:  # scalar
                return ()
            if b[p + 3] == 2:  # null
                return None
            q = p + 4
        else:
            raise H5Error(f"dataspace version {ver}")
        return tuple(self._u(q + 8 * i, 8) for i in range(rank))

    # -- groups ---------------------------------------------------------------------------------
    def _group_tables(self, hdr):
        for mtype, p, _n, _f in self._messages(hdr):
            if mtype == 0x11:
                return self._u(p, 8), self._u(p + 8, 8)
            if mtype in (0x02, 0x06):
                raise H5Error("new-style (link message) groups are not supported")
        return None

    def _children(self, hdr):
        tabs = self._group_tables(hdr)
        if tabs is None:
            raise H5Error("not a group")
        btree, heap = tabs
        heap_data = self._heap_data(heap)
        out = {}
        self._walk_group_btree(btree, heap_data, out)
        return out

    def _walk_group_btree(self, addr, heap_data, out):
        b = self.b
        if b[addr:addr + 4] != b"TREE" or b[addr + 4] != 0:
            raise H5Error(f"group B-tree node missing at {addr}")
        level, used = b[addr + 5], self._u(addr + 6, 2)
        p = addr + 24
        for i in range(used):
            child = self._u(p + 8, 8)  # key (heap offset), then child
            p += 16
            if level > 0:
                self._walk_group_btree(child, heap_data, out)
            else:
                if b[child:child + 4] != b"SNOD":
                    raise H5Error(f"symbol node missing at {child}")
                n = self._u(child + 6, 2)
                for k in range(n):
                    e = self._entry(child + 8 + 40 * k)
                    out[self._cstr(heap_data + e["name_off"])] = e["hdr"]

    def _resolve(self, path):
        hdr = self.root["hdr"]
        for part in [x for x in path.split("/") if x]:
            kids = self._children(hdr)
            if part not in kids:
                raise KeyError(f"{self.path}: no '{part}' in '{path}'")
            hdr = kids[part]
        return hdr

    def keys(self, path="/"):
        return sorted(self._children(self._resolve(path)))

    def is_group(self, path):
        return self._group_tables(self._resolve(path)) is not None

    def __contains__(self, path):
        try:
            self._resolve(path)
            return True
        except KeyError:
            return False

    # -- data -----------------------------------------------------------------------------------
    def _vlen_strings(self, raw, count):
        out = []
        for i in range(count):
            n = int.from_bytes(raw[16 * i:16 * i + 4], "little")
            coll = int.from_bytes(raw[16 * i + 4:16 * i + 12], "little")
            idx = int.from_bytes(raw[16 * i + 12:16 * i + 16], "little")
            out.append(self._gheap_object(coll, idx)[:n].decode())
        return out

    def _gheap_object(self, coll, idx):
        b = self.b
        if b[coll:coll + 4] != b"GCOL":
            raise H5Error(f"global heap collection missing at {coll}")
        size = self._u(coll + 8, 8)
        p, end = coll + 16, coll + size
        while p + 16 <= end:
            oi, osz = self._u(p, 2), self._u(p + 8, 8)
            if oi == 0:
                break
            if oi == idx:
                return b[p + 16:p + 16 + osz]
            p += 16 + (osz + 7) // 8 * 8
        raise H5Error(f"global heap object {idx} not found")

    def _convert(self, t, raw, shape):
        count = int(np.prod(shape)) if shape else 1
        if t.vlen_str:
            vals = self._vlen_strings(raw, count)
            return vals[0] if shape == () else np.array(vals, dtype=object).reshape(shape)
        a = np.frombuffer(raw, t.dtype, count).copy()
        if t.cls == 6 and a.dtype.names and set(a.dtype.names) == {"r", "i"}:
            a = a["r"].astype(np.float64) + 1j * a["i"].astype(np.float64)
        elif t.cls == 8 and set(t.enum.values()) == {"FALSE", "TRUE"}:
            a = a.astype(bool)
        elif t.cls == 3:
            a = np.array([x.split(b"\0")[0].decode() for x in a], dtype=object)
        elif t.cls in (0, 1):
            a = a.astype(a.dtype.newbyteorder("="))
        a = a.reshape(shape)
        return a[()] if shape == () else a

    def _dataset(self, hdr):
        t = shape = layout = None
        filters = []
        for mtype, p, n, _f in self._messages(hdr):
            if mtype == 0x01:
                shape = self._space(p)
            elif mtype == 0x03:
                t, _ = self._dtype(p)
            elif mtype == 0x08:
                layout = p
            elif mtype == 0x0B:
                filters = self._filters(p)
        if t is None or layout is None:
            raise H5Error("not a dataset")
        b = self.b
        ver, cls = b[layout], b[layout + 1]
        if ver != 3:
            raise H5Error(f"data layout version {ver}")
        count = int(np.prod(shape)) if shape else 1
        nbytes = count * t.size
        if cls == 0:
            size = self._u(layout + 2, 2)
            raw = b[layout + 4:layout + 4 + size]
        elif cls == 1:
            addr = self._u(layout + 2, 8)
            raw = bytes(nbytes) if addr == _UNDEF else b[addr:addr + nbytes]
        elif cls == 2:
            raw = self._chunked(layout, shape, t.size, filters)
        else:
            raise H5Error(f"layout class {cls}")
        if len(raw) < nbytes:
            raise H5Error("dataset storage shorter than its dataspace")
        return self._convert(t, raw[:nbytes], shape)

    def _filters(self, p):
        b = self.b
        ver, nf = b[p], b[p + 1]
        q = p + (8 if ver == 1 else 2)
        out = []
        for _ in range(nf):
            fid = self._u(q, 2)
            if ver == 1 or fid >= 256:
                nlen = self._u(q + 2, 2)
                ncv = self._u(q + 6, 2)
                q += 8 + ((nlen + 7) // 8 * 8 if ver == 1 else nlen)
            else:
                ncv = self._u(q + 6, 2) if ver == 1 else self._u(q + 4, 2)
                q += 6
            cvals = [self._u(q + 4 * i, 4) for i in range(ncv)]
            q += 4 * ncv
            if ver == 1 and ncv % 2:
                q += 4
            out.append((fid, cvals))
        return out

    def _chunked(self, layout, shape, esize, filters):
        b = self.b
        rank = b[layout + 2]  # dataspace rank + 1
        btree = self._u(layout + 3, 8)
        cdims = [self._u(layout + 11 + 4 * i, 4) for i in range(rank)]
        cshape = cdims[:-1]
        out = np.zeros(int(np.prod(shape)) * esize, np.uint8).reshape(tuple(shape) + (esize,))
        if btree == _UNDEF:
            return out.tobytes()
        for offs, size, mask, addr in self._chunk_list(btree, rank):
            raw = b[addr:addr + size]
            for k, (fid, cv) in reversed(list(enumerate(filters))):
                if mask & (1 << k):
                    continue
                if fid == 1:
                    raw = zlib.decompress(raw)
                elif fid == 2:
                    n = len(raw) // esize
                    raw = np.frombuffer(raw, np.uint8).reshape(esize, n).T.tobytes()
                else:
                    raise H5Error(f"filter {fid} not supported")
            chunk = np.frombuffer(raw, np.uint8)[:int(np.prod(cshape)) * esize].reshape(tuple(cshape) + (esize,))
            sl_out, sl_in = [], []
            for d in range(len(shape)):
                lo = offs[d]
                hi = min(lo + cshape[d], shape[d])
                sl_out.append(slice(lo, hi))
                sl_in.append(slice(0, hi - lo))
            out[tuple(sl_out)] = chunk[tuple(sl_in)]
        return out.tobytes()

    def _chunk_list(self, addr, rank):
        b = self.b
        if b[addr:addr + 4] != b"TREE" or b[addr + 4] != 1:
            raise H5Error(f"chunk B-tree node missing at {addr}")
        level, used = b[addr + 5], self._u(addr + 6, 2)
        ksz = 8 + 8 * rank
        p = addr + 24
        out = []
        for _ in range(used):
            size, mask = self._u(p, 4), self._u(p + 4, 4)
            offs = [self._u(p + 8 + 8 * i, 8) for i in range(rank)]
            child = self._u(p + ksz, 8)
            if level > 0:
                out += self._chunk_list(child, rank)
            else:
                out.append((offs, size, mask, child))
            p += ksz + 8
        return out

    def __getitem__(self, path):
        return self._dataset(self._resolve(path))

    def shape(self, path):
        for mtype, p, _n, _f in self._messages(self._resolve(path)):
            if mtype == 0x01:
                return self._space(p)
        raise H5Error(f"{path}: no dataspace")

    def attrs(self, path="/"):
        """The attributes of the object at path, by name."""
        out = {}
        b = self.b
        for mtype, p, _n, _f in self._messages(self._resolve(path)):
            if mtype != 0x0C:
                continue
            ver = b[p]
            nlen, tlen, slen = self._u(p + 2, 2), self._u(p + 4, 2), self._u(p + 6, 2)
            q = p + (9 if ver == 3 else 8)
            pad = (lambda n: (n + 7) // 8 * 8) if ver == 1 else (lambda n: n)
            name = b[q:q + nlen].split(b"\0")[0].decode()
            q += pad(nlen)
            t, _ = self._dtype(q)
            q += pad(tlen)
            shape = self._space(q)
            q += pad(slen)
            count = int(np.prod(shape)) if shape else 1
            raw = b[q:q + count * (16 if t.vlen_str else t.size)]
            out[name] = self._convert(t, raw, shape if shape is not None else ())
        return out
