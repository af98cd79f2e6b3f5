"""A minimal HDF5 writer for CPU tests of the HDF5 reader and the input loaders (test infrastructure).

It writes the subset of the published HDF5 file format that safire_b200.h5read reads, so that the
Hamiltonian and NOMSD trial loaders run on the CPU without the reference's own files:

  * a version 0 superblock (8-byte offsets and lengths) whose root is a symbol-table group;
  * groups as version 1 object headers holding a symbol-table message, each with one local heap
    (the member names), one version 1 B-tree leaf of type 0 and one symbol-table node;
  * datasets of little-endian int64 or float64 values of any rank, contiguous storage, with a
    version 1 dataspace and a version 3 layout message;
  * version 1 attributes: scalar float64 or int64, fixed-length strings.

Complex arrays go in with a trailing dimension of 2 (re, im), which the loaders accept.  It is not
a general HDF5 writer: no fill-value or modification-time messages, at most 64 members per group.

    write(path, {"Hamiltonian/hcore": h, "Hamiltonian/DenseFactorized/L": L},
          attrs={"Hamiltonian": {"nuclear_energy": 1.5}})
"""
import struct

import numpy as np

_SIG = b"\x89HDF\r\n\x1a\n"
_UNDEF = 0xFFFFFFFFFFFFFFFF
_LEAF_K = 32      # group leaf node K: up to 2K members in a symbol-table node
_INTERNAL_K = 16  # group internal node K (sizes the B-tree node)


def _pad8(b):
    return b + b"\0" * (-len(b) % 8)


def _dtype_msg(a):
    """Datatype message body for an int64, float64 or fixed-length string value."""
    if a.dtype.kind == "S":
        return struct.pack("<BBBBI", 0x13, 0, 0, 0, a.dtype.itemsize)
    if a.dtype.kind in "iu":
        # fixed point, version 1: little endian, signed; bit offset 0, precision 64
        return struct.pack("<BBBBIHH", 0x10, 0x08, 0, 0, 8, 0, 64)
    if a.dtype.kind == "f":
        # floating point, version 1: little endian, implied leading mantissa bit (normalization 2),
        # sign at bit 63; bit offset 0, precision 64, exponent at 52 (11 bits), mantissa at 0
        # (52 bits), exponent bias 1023
        return struct.pack("<BBBBIHHBBBBI", 0x11, 0x20, 63, 0, 8, 0, 64, 52, 11, 0, 52, 1023)
    raise ValueError(f"dtype {a.dtype} is not written")


def _canonical(v):
    a = np.asarray(v)
    if a.dtype.kind == "U":
        a = np.char.encode(a, "ascii")
        a = a.astype(f"S{max(1, a.dtype.itemsize) + 1}")  # room for the terminating null
    elif a.dtype.kind == "b" or a.dtype.kind in "iu":
        a = a.astype("<i8")
    elif a.dtype.kind == "f":
        a = a.astype("<f8")
    elif a.dtype.kind == "c":
        raise ValueError("complex values go in as a trailing dimension of 2")
    elif a.dtype.kind != "S":
        raise ValueError(f"dtype {a.dtype} is not written")
    return a


def _space_msg(shape):
    """Dataspace message, version 1 (rank 0: a scalar)."""
    return struct.pack("<BBBBI", 1, len(shape), 0, 0, 0) + b"".join(struct.pack("<Q", d) for d in shape)


def _message(mtype, body):
    body = _pad8(body)
    return struct.pack("<HHBBBB", mtype, len(body), 0, 0, 0, 0) + body


def _attribute(name, value):
    a = _canonical(value)
    nm = name.encode() + b"\0"
    dt = _dtype_msg(a)
    sp = _space_msg(a.shape)
    body = struct.pack("<BBHHH", 1, 0, len(nm), len(dt), len(sp)) + _pad8(nm) + _pad8(dt) + _pad8(sp)
    return _message(0x0C, body + a.tobytes())


class _Writer:
    def __init__(self):
        self.buf = bytearray(96)  # the superblock, written last

    def alloc(self, data):
        self.buf += b"\0" * (-len(self.buf) % 8)
        at = len(self.buf)
        self.buf += data
        return at

    def header(self, messages):
        body = b"".join(messages)
        return self.alloc(struct.pack("<BBHII", 1, 0, len(messages), 1, len(body)) + b"\0" * 4 + body)

    def dataset(self, value, attrs):
        a = _canonical(value)
        data = a.tobytes()
        at = self.alloc(data) if data else _UNDEF
        layout = struct.pack("<BBQQ", 3, 1, at, len(data))
        msgs = [_message(0x01, _space_msg(a.shape)), _message(0x03, _dtype_msg(a)), _message(0x08, layout)]
        msgs += [_attribute(k, v) for k, v in attrs.items()]
        return self.header(msgs)

    def group(self, members, attrs):
        """members: name -> object header address."""
        names = sorted(members)
        if len(names) > 2 * _LEAF_K:
            raise ValueError(f"{len(names)} members in one group (at most {2 * _LEAF_K})")
        heap, offs = b"\0" * 8, {}
        for n in names:
            offs[n] = len(heap)
            heap += _pad8(n.encode() + b"\0")
        heap_data = self.alloc(heap)
        heap_at = self.alloc(b"HEAP" + struct.pack("<B3xQQQ", 0, len(heap), _UNDEF, heap_data))
        snod = b"SNOD" + struct.pack("<BBH", 1, 0, len(names))
        for n in names:
            snod += struct.pack("<QQI4x16x", offs[n], members[n], 0)
        snod += b"\0" * (40 * (2 * _LEAF_K - len(names)))
        snod_at = self.alloc(snod)
        # one leaf: key 0 (the empty name), the symbol node, key of the node's last name
        tree = b"TREE" + struct.pack("<BBHQQ", 0, 0, 1, _UNDEF, _UNDEF)
        tree += struct.pack("<QQQ", 0, snod_at, offs[names[-1]] if names else 0)
        tree += b"\0" * (8 * (4 * _INTERNAL_K + 1) - 24)
        tree_at = self.alloc(tree)
        msgs = [_message(0x11, struct.pack("<QQ", tree_at, heap_at))]
        msgs += [_attribute(k, v) for k, v in attrs.items()]
        return self.header(msgs), tree_at, heap_at


def write(path, datasets, attrs=None):
    """Write the datasets (path -> array) and attributes (object path -> {name: value}) to path;
    the groups on the paths are made as needed."""
    attrs = {k.strip("/"): v for k, v in (attrs or {}).items()}
    tree = {}
    for p, v in datasets.items():
        parts = [x for x in p.split("/") if x]
        node = tree
        for g in parts[:-1]:
            node = node.setdefault(g, {})
            if not isinstance(node, dict):
                raise ValueError(f"{p}: {g} is a dataset")
        node[parts[-1]] = v
    for p in attrs:  # groups that only carry attributes
        node = tree
        for g in [x for x in p.split("/") if x]:
            node = node.setdefault(g, {})
    w = _Writer()

    def emit(node, where):
        members = {}
        for name, v in node.items():
            sub = f"{where}/{name}".strip("/")
            if isinstance(v, dict):
                members[name] = emit(v, sub)[0]
            else:
                members[name] = w.dataset(v, attrs.get(sub, {}))
        return w.group(members, attrs.get(where, {}))

    root_hdr, root_tree, root_heap = emit(tree, "")
    sb = _SIG + struct.pack("<BBBBBBBB", 0, 0, 0, 0, 0, 8, 8, 0)
    sb += struct.pack("<HHI", _LEAF_K, _INTERNAL_K, 0)
    sb += struct.pack("<QQQQ", 0, _UNDEF, len(w.buf), _UNDEF)
    sb += struct.pack("<QQI4xQQ", 0, root_hdr, 1, root_tree, root_heap)
    assert len(sb) == 96
    w.buf[:96] = sb
    with open(path, "wb") as f:
        f.write(bytes(w.buf))
