"""The .NET binary serialization stream (MS-NRBF), as icFlow's snapshots use it.

icFlow's mesh frames end with two objects written by .NET's BinaryFormatter
(v3Library/Geometry/Mesh/Mesh.cs:257-260): the mesh's `List<SurfaceFragment>`
and its `TranslationCollection`.  A frame file is read past them, and written
with them, through this module.  It follows Microsoft's published [MS-NRBF]
record grammar: a serialization header, class records with their member
type information, arrays, strings, references, null runs and the message end.

`read(buf, pos)` parses one serialized object graph starting at `pos` and
returns (root, end).  Classes come back as `NrbfObject` (type name and an
ordered dict of members), arrays as Python lists, strings as str, primitives
as int/float/bool; references are resolved.  `Writer` emits the record shapes
BinaryFormatter uses for the classes icFlow stores (a class with members and
their types, `ClassWithId` for repeats, single-dimension arrays, the
`System.Collections.Generic.List` layout).  Neither direction was run against
a .NET runtime (none is available here): the reader is checked on streams of
the spec's grammar, the writer by reading its output back.
"""
from __future__ import annotations

import struct
from dataclasses import dataclass, field

# RecordTypeEnumeration
HEADER, CLASS_WITH_ID, SYS_CLASS_MEMBERS, CLASS_MEMBERS, SYS_CLASS_MEMBERS_TYPES, CLASS_MEMBERS_TYPES = 0, 1, 2, 3, 4, 5
OBJECT_STRING, BINARY_ARRAY, MEMBER_PRIMITIVE, MEMBER_REFERENCE, OBJECT_NULL, MESSAGE_END = 6, 7, 8, 9, 10, 11
LIBRARY, NULL_MULTIPLE_256, NULL_MULTIPLE, ARRAY_PRIMITIVE, ARRAY_OBJECT, ARRAY_STRING = 12, 13, 14, 15, 16, 17

# BinaryTypeEnumeration
BT_PRIMITIVE, BT_STRING, BT_OBJECT, BT_SYSTEM_CLASS, BT_CLASS, BT_OBJECT_ARRAY, BT_STRING_ARRAY, BT_PRIMITIVE_ARRAY = range(8)

# PrimitiveTypeEnumeration -> struct format (Decimal travels as a string)
P_BOOLEAN, P_BYTE, P_CHAR, P_DECIMAL, P_DOUBLE, P_INT16, P_INT32, P_INT64 = 1, 2, 3, 5, 6, 7, 8, 9
P_SBYTE, P_SINGLE, P_TIMESPAN, P_DATETIME, P_UINT16, P_UINT32, P_UINT64, P_NULL, P_STRING = range(10, 19)
_PRIM = {P_BOOLEAN: "<?", P_BYTE: "<B", P_DOUBLE: "<d", P_INT16: "<h", P_INT32: "<i", P_INT64: "<q", P_SBYTE: "<b",
         P_SINGLE: "<f", P_TIMESPAN: "<q", P_DATETIME: "<Q", P_UINT16: "<H", P_UINT32: "<I", P_UINT64: "<Q"}

MSCORLIB = "mscorlib, Version=4.0.0.0, Culture=neutral, PublicKeyToken=b77a5c561934e089"


class NrbfError(ValueError):
    pass


@dataclass
class NrbfObject:
    type_name: str
    members: dict = field(default_factory=dict)
    library: str | None = None

    def __getitem__(self, k):
        return self.members[k]

    def member(self, suffix: str):
        """The member whose name is `suffix` or ends with it (an auto
        property's backing field "<x>k__BackingField", a base class's
        "List`1+_items")."""
        for k, v in self.members.items():
            if k == suffix or k.endswith(suffix):
                return v
        raise KeyError(suffix)


class _Ref:
    __slots__ = ("id",)

    def __init__(self, i):
        self.id = i


class _Nulls:
    __slots__ = ("n",)

    def __init__(self, n):
        self.n = n


class _Reader:
    def __init__(self, buf: bytes, pos: int):
        self.b = buf
        self.p = pos
        self.objs: dict[int, object] = {}
        self.meta: dict[int, tuple] = {}  # object id -> (name, members, types, infos, library)
        self.libs: dict[int, str] = {}

    def take(self, fmt):
        n = struct.calcsize(fmt)
        if self.p + n > len(self.b):
            raise NrbfError("stream ends inside a record")
        v = struct.unpack_from(fmt, self.b, self.p)[0]
        self.p += n
        return v

    def string(self) -> str:
        # LengthPrefixedString: 7-bit encoded length, UTF-8
        n, shift = 0, 0
        for _ in range(5):
            c = self.take("<B")
            n |= (c & 0x7F) << shift
            shift += 7
            if not c & 0x80:
                break
        else:
            raise NrbfError("bad string length")
        if self.p + n > len(self.b):
            raise NrbfError("stream ends inside a string")
        s = self.b[self.p:self.p + n].decode("utf-8")
        self.p += n
        return s

    def prim(self, t):
        if t == P_CHAR:  # one UTF-8 character
            c = self.b[self.p]
            n = 1 if c < 0x80 else (2 if c < 0xE0 else (3 if c < 0xF0 else 4))
            s = self.b[self.p:self.p + n].decode("utf-8")
            self.p += n
            return s
        if t in (P_DECIMAL, P_STRING):
            return self.string()
        if t == P_NULL:
            return None
        if t not in _PRIM:
            raise NrbfError(f"unknown primitive type {t}")
        return self.take(_PRIM[t])

    def class_info(self):
        oid = self.take("<i")
        name = self.string()
        n = self.take("<i")
        if n < 0:
            raise NrbfError("negative member count")
        members = [self.string() for _ in range(n)]
        return oid, name, members

    def type_info(self, n):
        types = [self.take("<B") for _ in range(n)]
        infos = []
        for t in types:
            if t in (BT_PRIMITIVE, BT_PRIMITIVE_ARRAY):
                infos.append(self.take("<B"))
            elif t == BT_SYSTEM_CLASS:
                infos.append(self.string())
            elif t == BT_CLASS:
                infos.append((self.string(), self.take("<i")))
            elif t in (BT_STRING, BT_OBJECT, BT_OBJECT_ARRAY, BT_STRING_ARRAY):
                infos.append(None)
            else:
                raise NrbfError(f"unknown binary type {t}")
        return types, infos

    def members(self, oid, name, members, types, infos, lib):
        obj = NrbfObject(name, {}, self.libs.get(lib) if lib is not None else None)
        self.objs[oid] = obj
        for m, t, info in zip(members, types, infos):
            if t == BT_PRIMITIVE:
                obj.members[m] = self.prim(info)
            else:
                obj.members[m] = self.value()
        return obj

    def value(self):
        """One record standing for a value (an object, a reference, a null)."""
        while True:
            rt = self.take("<B")
            if rt == LIBRARY:
                lid = self.take("<i")
                self.libs[lid] = self.string()
                continue
            return self.record(rt)

    def record(self, rt):
        if rt == CLASS_WITH_ID:
            oid, mid = self.take("<i"), self.take("<i")
            if mid not in self.meta:
                raise NrbfError(f"class metadata {mid} not seen")
            name, members, types, infos, lib = self.meta[mid]
            return self.members(oid, name, members, types, infos, lib)
        if rt in (CLASS_MEMBERS_TYPES, SYS_CLASS_MEMBERS_TYPES):
            oid, name, members = self.class_info()
            types, infos = self.type_info(len(members))
            lib = self.take("<i") if rt == CLASS_MEMBERS_TYPES else None
            self.meta[oid] = (name, members, types, infos, lib)
            return self.members(oid, name, members, types, infos, lib)
        if rt in (CLASS_MEMBERS, SYS_CLASS_MEMBERS):
            # members without type information: each value is a record
            oid, name, members = self.class_info()
            lib = self.take("<i") if rt == CLASS_MEMBERS else None
            types = [BT_OBJECT] * len(members)
            infos = [None] * len(members)
            self.meta[oid] = (name, members, types, infos, lib)
            return self.members(oid, name, members, types, infos, lib)
        if rt == OBJECT_STRING:
            oid = self.take("<i")
            s = self.string()
            self.objs[oid] = s
            return s
        if rt == MEMBER_PRIMITIVE:
            return self.prim(self.take("<B"))
        if rt == MEMBER_REFERENCE:
            return _Ref(self.take("<i"))
        if rt == OBJECT_NULL:
            return None
        if rt == NULL_MULTIPLE_256:
            return _Nulls(self.take("<B"))
        if rt == NULL_MULTIPLE:
            return _Nulls(self.take("<i"))
        if rt == ARRAY_PRIMITIVE:
            oid, n, t = self.take("<i"), self.take("<i"), self.take("<B")
            if n < 0:
                raise NrbfError(f"bad array length {n}")
            if t in _PRIM and t != P_CHAR:
                fmt = _PRIM[t][1]
                size = struct.calcsize("<" + fmt)
                if self.p + n * size > len(self.b):
                    raise NrbfError("stream ends inside an array")
                arr = list(struct.unpack_from(f"<{n}{fmt}", self.b, self.p))
                self.p += n * size
            else:
                arr = [self.prim(t) for _ in range(n)]
            self.objs[oid] = arr
            return arr
        if rt in (ARRAY_OBJECT, ARRAY_STRING):
            oid, n = self.take("<i"), self.take("<i")
            arr = self.elements(n, BT_OBJECT, None)
            self.objs[oid] = arr
            return arr
        if rt == BINARY_ARRAY:
            oid = self.take("<i")
            kind = self.take("<B")
            rank = self.take("<i")
            lens = [self.take("<i") for _ in range(rank)]
            if kind in (3, 4, 5):
                for _ in range(rank):
                    self.take("<i")  # lower bounds
            t = self.take("<B")
            info = None
            if t in (BT_PRIMITIVE, BT_PRIMITIVE_ARRAY):
                info = self.take("<B")
            elif t == BT_SYSTEM_CLASS:
                info = self.string()
            elif t == BT_CLASS:
                info = (self.string(), self.take("<i"))
            total = 1
            for n in lens:
                if n < 0:
                    raise NrbfError(f"bad array length {n}")
                total *= n
            arr = self.elements(total, t, info)
            self.objs[oid] = arr
            return arr
        if rt == HEADER:
            raise NrbfError("second header inside a stream")
        raise NrbfError(f"unsupported record type {rt}")

    def elements(self, n, t, info):
        if n < 0 or n > len(self.b):  # every element takes at least one byte
            raise NrbfError(f"bad array length {n}")
        out = []
        while len(out) < n:
            if t == BT_PRIMITIVE:
                out.append(self.prim(info))
                continue
            v = self.value()
            if isinstance(v, _Nulls):
                if v.n < 0 or len(out) + v.n > n:
                    raise NrbfError("null run past the end of an array")
                out.extend([None] * v.n)
            else:
                out.append(v)
        return out

    def resolve(self, v, seen):
        if isinstance(v, _Ref):
            if v.id not in self.objs:
                raise NrbfError(f"reference to unknown object {v.id}")
            return self.resolve(self.objs[v.id], seen)
        if isinstance(v, NrbfObject):
            if id(v) not in seen:
                seen.add(id(v))
                for k in v.members:
                    v.members[k] = self.resolve(v.members[k], seen)
            return v
        if isinstance(v, list):
            if id(v) not in seen:
                seen.add(id(v))
                for i in range(len(v)):
                    v[i] = self.resolve(v[i], seen)
            return v
        return v


def read(buf: bytes, pos: int = 0):
    """Parses one object graph from `buf` at `pos`; returns (root, end)."""
    r = _Reader(buf, pos)
    if r.take("<B") != HEADER:
        raise NrbfError("no serialization header")
    root, _hid, major, _minor = r.take("<i"), r.take("<i"), r.take("<i"), r.take("<i")
    if major != 1:
        raise NrbfError(f"unsupported stream version {major}")
    while True:
        rt = r.take("<B")
        if rt == MESSAGE_END:
            break
        if rt == LIBRARY:
            lid = r.take("<i")
            r.libs[lid] = r.string()
            continue
        r.record(rt)
    if root not in r.objs:
        raise NrbfError("root object missing")
    return r.resolve(r.objs[root], set()), r.p


def list_items(obj) -> list:
    """The elements of a serialized System.Collections.Generic.List (or a
    class derived from it): its _items array cut to _size."""
    if obj is None:
        return []
    items = obj.member("_items")
    n = obj.member("_size")
    return list(items[:n]) if items is not None else []


class Writer:
    """Emits one object graph in BinaryFormatter's record shapes.

    Object ids are the caller's (new_id), so that a member can reference an
    object written after it, as BinaryFormatter does.  A member is
    (name, binary type, additional info, value): for BT_PRIMITIVE the value
    itself; otherwise an object id (a MemberReference), None (ObjectNull) or
    a callable that writes the value's record inline."""

    def __init__(self, library: str):
        self.out = bytearray()
        self.next_id = 1
        self.library = library
        self.lib_id = None
        self.meta: dict[str, int] = {}  # class name -> id of its first record

    def _b(self, fmt, v):
        self.out += struct.pack(fmt, v)

    def _s(self, s: str):
        data = s.encode("utf-8")
        n = len(data)
        while True:
            c = n & 0x7F
            n >>= 7
            self.out.append(c | (0x80 if n else 0))
            if not n:
                break
        self.out += data

    def new_id(self) -> int:
        i = self.next_id
        self.next_id += 1
        return i

    def lib(self) -> int:
        """The library's id; its record is written on first use."""
        if self.lib_id is None:
            self.lib_id = self.new_id()
            self._b("<B", LIBRARY)
            self._b("<i", self.lib_id)
            self._s(self.library)
        return self.lib_id

    def begin(self, root: int = 1):
        self._b("<B", HEADER)
        self._b("<i", root)
        self._b("<i", -1)
        self._b("<i", 1)
        self._b("<i", 0)

    def end(self) -> bytes:
        self._b("<B", MESSAGE_END)
        return bytes(self.out)

    def class_record(self, oid: int, name: str, members: list, system: bool = False):
        if not system or any(m[1] == BT_CLASS for m in members):
            lib = self.lib()
        if name in self.meta:
            self._b("<B", CLASS_WITH_ID)
            self._b("<i", oid)
            self._b("<i", self.meta[name])
        else:
            self.meta[name] = oid
            self._b("<B", SYS_CLASS_MEMBERS_TYPES if system else CLASS_MEMBERS_TYPES)
            self._b("<i", oid)
            self._s(name)
            self._b("<i", len(members))
            for m in members:
                self._s(m[0])
            for m in members:
                self._b("<B", m[1])
            for m in members:
                bt, info = m[1], m[2]
                if bt in (BT_PRIMITIVE, BT_PRIMITIVE_ARRAY):
                    self._b("<B", info)
                elif bt == BT_SYSTEM_CLASS:
                    self._s(info)
                elif bt == BT_CLASS:
                    self._s(info)
                    self._b("<i", lib)
            if not system:
                self._b("<i", lib)
        for m in members:
            bt, info, v = m[1], m[2], m[3]
            if bt == BT_PRIMITIVE:
                self._b(_PRIM[info], v)
            elif v is None:
                self._b("<B", OBJECT_NULL)
            elif callable(v):
                v()
            else:
                self._b("<B", MEMBER_REFERENCE)
                self._b("<i", v)

    def primitive_array(self, oid: int, t: int, values):
        self._b("<B", ARRAY_PRIMITIVE)
        self._b("<i", oid)
        self._b("<i", len(values))
        self._b("<B", t)
        fmt = _PRIM[t]
        for v in values:
            self._b(fmt, v)

    def class_array(self, oid: int, elem_type: str, refs: list, length: int):
        """A single-dimension array of class elements of the library:
        references to `refs`, then nulls up to `length`."""
        lib = self.lib()
        self._b("<B", BINARY_ARRAY)
        self._b("<i", oid)
        self._b("<B", 0)  # single
        self._b("<i", 1)
        self._b("<i", length)
        self._b("<B", BT_CLASS)
        self._s(elem_type)
        self._b("<i", lib)
        for r in refs:
            self._b("<B", MEMBER_REFERENCE)
            self._b("<i", r)
        n = length - len(refs)
        if n == 1:
            self._b("<B", OBJECT_NULL)
        elif 1 < n < 256:
            self._b("<B", NULL_MULTIPLE_256)
            self._b("<B", n)
        elif n >= 256:
            self._b("<B", NULL_MULTIPLE)
            self._b("<i", n)
