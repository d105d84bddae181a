"""Test infrastructure: a reader for GSD 2.0 files, the container of the HOOMD-blue GSD
library that the reference vendors (src/gsd.c, src/gsd.h) and writes its trajectory with
(PS_Box_gsdUtils.cu:14-168).  The tests read the B200 library's trajectories with it and
pin it against the reference's own reader (oracle/ref_harness/gsd_dump.c, linked with the
reference's gsd.c).

Layout (gsd.h:124-187, format version 2.0): a 256-byte header {u64 magic 0x65DF65DF65DF65DF,
u64 index_location, u64 index_allocated_entries, u64 namelist_location,
u64 namelist_allocated_entries (x 64 bytes), u32 schema_version, u32 gsd_version,
char application[64], char schema[64], char reserved[80]}; an index of 32-byte entries
{u64 frame, u64 N, i64 location, u32 M, u16 id, u8 type, u8 flags} sorted by (frame, id)
and ended by the first entry with location 0; a namelist of NUL-terminated names (id = rank).
The checks follow the reader's (gsd.c:421-458 entry validity, :1440-1560 header and
namelist): a file failing one raises ValueError.
"""
import struct

import numpy as np

MAGIC = 0x65DF65DF65DF65DF
TYPES = {1: np.uint8, 2: np.uint16, 3: np.uint32, 4: np.uint64, 5: np.int8, 6: np.int16, 7: np.int32,
         8: np.int64, 9: np.float32, 10: np.float64}
HEADER = struct.Struct("<QQQQQII64s64s80s")
ENTRY = struct.Struct("<QQqIHBB")


def version(major, minor):
    return (major << 16) | minor


class GsdFile:
    def __init__(self, path):
        self.raw = open(path, "rb").read()
        if len(self.raw) < HEADER.size:
            raise ValueError("not a GSD file: too short")
        (magic, self.index_location, self.index_allocated, self.namelist_location, self.namelist_allocated,
         self.schema_version, self.gsd_version, app, schema, _) = HEADER.unpack_from(self.raw, 0)
        if magic != MAGIC:
            raise ValueError("not a GSD file: bad magic")
        if not (version(1, 0) <= self.gsd_version < version(3, 0)):
            raise ValueError("unsupported GSD file version %#x" % self.gsd_version)
        self.application = app.split(b"\0", 1)[0].decode()
        self.schema = schema.split(b"\0", 1)[0].decode()
        size = len(self.raw)
        nl_bytes = 64 * self.namelist_allocated
        if self.namelist_location + nl_bytes > size:
            raise ValueError("corrupt: namelist outside the file")
        nl = self.raw[self.namelist_location:self.namelist_location + nl_bytes]
        if nl_bytes == 0 or nl[-1] != 0:
            raise ValueError("corrupt: namelist not terminated")
        self.names = []
        pos = 0
        while pos < nl_bytes and nl[pos] != 0:
            end = nl.index(b"\0", pos)
            self.names.append(nl[pos:end].decode())
            pos = end + 1 if self.gsd_version >= version(2, 0) else pos + 64
        if self.index_location + 32 * self.index_allocated > size:
            raise ValueError("corrupt: index outside the file")
        self.entries = []
        for k in range(self.index_allocated):
            e = ENTRY.unpack_from(self.raw, self.index_location + 32 * k)
            frame, N, loc, M, eid, typ, flags = e
            if loc == 0:
                break
            if typ not in TYPES:
                raise ValueError("corrupt: entry %d has type %d" % (k, typ))
            if loc + N * M * np.dtype(TYPES[typ]).itemsize > size:
                raise ValueError("corrupt: entry %d data past the end of the file" % k)
            if frame >= self.index_allocated:
                raise ValueError("corrupt: entry %d frame %d >= index capacity" % (k, frame))
            if eid >= len(self.names):
                raise ValueError("corrupt: entry %d name id %d" % (k, eid))
            if flags != 0:
                raise ValueError("corrupt: entry %d flags" % k)
            if self.entries and (frame, eid) <= (self.entries[-1][0], self.entries[-1][4]):
                raise ValueError("corrupt: index not sorted by (frame, id) at entry %d" % k)
            self.entries.append(e)
        self.nframes = self.entries[-1][0] + 1 if self.entries else 0

    def frame(self, f):
        """dict name -> array of frame f ((N,) when M == 1, else (N, M))."""
        out = {}
        for frame, N, loc, M, eid, typ, _ in self.entries:
            if frame != f:
                continue
            dt = np.dtype(TYPES[typ])
            a = np.frombuffer(self.raw, dtype=dt, count=N * M, offset=loc).copy()
            out[self.names[eid]] = a if M == 1 else a.reshape(N, M)
        return out

    def chunk_order(self, f):
        """(name, N, M, type) of frame f in index order."""
        return [(self.names[e[4]], e[1], e[3], e[5]) for e in self.entries if e[0] == f]
