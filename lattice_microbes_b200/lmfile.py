"""Reader for Lattice Microbes `.lm` files (HDF5), with no HDF5 library.

A `.lm` file is an HDF5 file behind a 512-byte user block that starts with
"LMH5" (io/SimulationFile_create.cpp:56-131), laid out as the reference's
docs/HDF5FileFormat.text describes: /Parameters (string attributes, double in
format 2), /Model/Reaction, /Model/Diffusion, and per replicate
/Simulations/%07d with SpeciesCounts, SpeciesCountTimes, LatticeTimes,
Lattice/%010d, SiteTimes, Sites/%010d, MaxParticleCounts and MaxSiteCounts
(io/SimulationFile.cpp:1166-1433, 2140-2230, 2368-2393).

This module reads the part of the HDF5 file format that libhdf5 writes for
such files with its default (1.8-compatible) settings, following the
published HDF5 File Format Specification: superblock versions 0 and 1,
version-1 object headers with continuation blocks, groups held in a symbol
table (version-1 B-tree of type 0, symbol-table nodes, local heap), simple and
scalar dataspaces, fixed-point, floating-point and fixed-length string types,
compact, contiguous and chunked layouts (version-1 B-tree of type 1), the
deflate, shuffle and Fletcher-32 filters, and version 1-3 attribute messages.
Anything else raises `H5FormatError` rather than being guessed at.
"""
import mmap
import os
import zlib

import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF
SIGNATURE = b"\x89HDF\r\n\x1a\n"


class H5FormatError(ValueError):
    """The file uses a part of the HDF5 format this reader does not read, or
    is not well formed."""


def _u(b, off, n):
    return int.from_bytes(b[off:off + n], "little")


class Dataset:
    def __init__(self, f, name, msgs):
        self.file, self.name = f, name
        self.shape, self.maxshape = None, None
        self.dtype = None
        self.layout = None
        self.filters = []
        self.attrs = {}
        for mtype, data in msgs:
            if mtype == 0x0001:
                self.shape, self.maxshape = f._dataspace(data, 0)
            elif mtype == 0x0003:
                self.dtype = f._datatype(data, 0)[0]
            elif mtype == 0x0008:
                self.layout = f._layout(data)
            elif mtype == 0x000B:
                self.filters = f._filters(data)
            elif mtype == 0x000C:
                k, v = f._attribute(data)
                self.attrs[k] = v
        if self.shape is None or self.dtype is None or self.layout is None:
            raise H5FormatError("dataset %s lacks a dataspace, datatype or layout" % name)

    def read(self):
        return self.file._read_dataset(self)

    @property
    def chunks(self):
        return tuple(self.layout[2]) if self.layout[0] == 2 else None


class Group:
    def __init__(self, f, name, msgs):
        self.file, self.name = f, name
        self.attrs = {}
        self.stab = None
        for mtype, data in msgs:
            if mtype == 0x0011:
                self.stab = (_u(data, 0, f.so), _u(data, f.so, f.so))
            elif mtype == 0x000C:
                k, v = f._attribute(data)
                self.attrs[k] = v
            elif mtype in (0x0002, 0x0006, 0x000A):
                raise H5FormatError("group %s uses link messages (new-style group)" % name)
        self._children = None

    def keys(self):
        return list(self._entries().keys())

    def _entries(self):
        if self._children is None:
            self._children = self.file._group_entries(*self.stab) if self.stab else {}
        return self._children

    def __contains__(self, key):
        try:
            self[key]
            return True
        except KeyError:
            return False

    def __getitem__(self, path):
        node = self
        for part in [p for p in path.split("/") if p]:
            if not isinstance(node, Group):
                raise KeyError(path)
            addr = node._entries().get(part)
            if addr is None:
                raise KeyError(path)
            node = node.file._object(addr, node.name.rstrip("/") + "/" + part)
        return node


class H5File:
    """A read-only HDF5 file (the subset in the module docstring)."""

    def __init__(self, path):
        self.path = path
        self._fh = open(path, "rb")
        size = os.fstat(self._fh.fileno()).st_size
        if size == 0:
            raise H5FormatError("%s is empty" % path)
        self.b = mmap.mmap(self._fh.fileno(), 0, access=mmap.ACCESS_READ)
        self.size = size
        self.sb = self._find_superblock(size)
        self._parse_superblock()
        self.root = self._object(self.root_addr, "/")

    def close(self):
        self.b.close()
        self._fh.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __getitem__(self, path):
        return self.root[path]

    # -- superblock ---------------------------------------------------------
    def _find_superblock(self, size):
        off = 0
        while off + 8 <= size:
            if self.b[off:off + 8] == SIGNATURE:
                return off
            off = 512 if off == 0 else off * 2
        raise H5FormatError("no HDF5 signature in %s" % self.path)

    def _parse_superblock(self):
        b, s = self.b, self.sb
        ver = b[s + 8]
        if ver not in (0, 1):
            raise H5FormatError("superblock version %d" % ver)
        self.so, self.sl = b[s + 13], b[s + 14]
        if (self.so, self.sl) != (8, 8):
            raise H5FormatError("offset/length sizes %d/%d" % (self.so, self.sl))
        self.leaf_k = _u(b, s + 16, 2)
        self.internal_k = _u(b, s + 18, 2)
        p = s + 24
        if ver == 1:
            self.istore_k = _u(b, p, 2)
            p += 4
        else:
            self.istore_k = 32
        self.base = _u(b, p, 8)
        self.eof = _u(b, p + 16, 8)
        if self.base != s:
            raise H5FormatError("base address %d for a superblock at %d" % (self.base, s))
        if self.eof > self.size:
            raise H5FormatError("truncated file: end of file %d > size %d" % (self.eof, self.size))
        entry = p + 32
        self.root_addr = _u(b, entry + 8, 8)
        self.userblock = bytes(b[:s])

    def _addr(self, a):
        if a == UNDEF:
            raise H5FormatError("undefined address")
        return self.base + a

    # -- object headers -----------------------------------------------------
    def _messages(self, addr):
        b = self.b
        p = self._addr(addr)
        if b[p] != 1:
            raise H5FormatError("object header version %d at %d" % (b[p], addr))
        nmsgs = _u(b, p + 2, 2)
        size = _u(b, p + 8, 4)
        blocks = [(p + 16, size)]
        out = []
        seen = 0
        while blocks:
            q, length = blocks.pop(0)
            end = q + length
            if end > self.size:
                raise H5FormatError("object header block past the end of the file")
            while q + 8 <= end:
                mtype, msize, flags = _u(b, q, 2), _u(b, q + 2, 2), b[q + 4]
                data = bytes(b[q + 8:q + 8 + msize])
                seen += 1
                if q + 8 + msize > end or msize % 8:
                    raise H5FormatError("message of %d bytes misaligned or past its header block" % msize)
                if flags & 0x02:
                    raise H5FormatError("shared message")
                if mtype == 0x0010:
                    blocks.append((self._addr(_u(data, 0, 8)), _u(data, 8, 8)))
                elif mtype != 0x0000:
                    out.append((mtype, data))
                q += 8 + msize
        if seen != nmsgs:
            raise H5FormatError("object header at %d holds %d messages, says %d" % (addr, seen, nmsgs))
        return out

    def _object(self, addr, name):
        msgs = self._messages(addr)
        types = {m for m, _ in msgs}
        if 0x0008 in types:
            return Dataset(self, name, msgs)
        return Group(self, name, msgs)

    # -- groups -------------------------------------------------------------
    def _heap(self, addr):
        b, p = self.b, self._addr(addr)
        if b[p:p + 4] != b"HEAP":
            raise H5FormatError("no local heap at %d" % addr)
        size = _u(b, p + 8, 8)
        free = _u(b, p + 16, 8)
        if free != 1 and free >= size:  # 1: no free block (libhdf5's H5HL_FREE_NULL)
            raise H5FormatError("local heap free list at %d of %d bytes" % (free, size))
        data = self._addr(_u(b, p + 24, 8))
        if data + size > self.size:
            raise H5FormatError("local heap past the end of the file")
        return bytes(b[data:data + size])

    @staticmethod
    def _cstr(heap, off):
        end = heap.index(b"\0", off)
        return heap[off:end].decode()

    def _group_entries(self, btree, heap_addr):
        heap = self._heap(heap_addr)
        out = {}
        for snod in self._btree_children(btree, 0):
            b, p = self.b, self._addr(snod)
            if b[p:p + 4] != b"SNOD":
                raise H5FormatError("no symbol table node at %d" % snod)
            n = _u(b, p + 6, 2)
            if n > 2 * self.leaf_k or p + 8 + 80 * self.leaf_k > self.size:
                raise H5FormatError("symbol table node at %d: %d entries or short" % (snod, n))
            for i in range(n):
                e = p + 8 + 40 * i
                out[self._cstr(heap, _u(b, e, 8))] = _u(b, e + 8, 8)
        return out

    def _btree_children(self, addr, node_type, rank=0):
        """Level-0 children of a version-1 B-tree, in key order; for raw-data
        trees (type 1) each child comes with its key (size, mask, offsets)."""
        if addr == UNDEF:
            return []
        b, p = self.b, self._addr(addr)
        if b[p:p + 4] != b"TREE" or b[p + 4] != node_type:
            raise H5FormatError("no B-tree node of type %d at %d" % (node_type, addr))
        level, used = b[p + 5], _u(b, p + 6, 2)
        ksize = 8 if node_type == 0 else 8 + 8 * (rank + 1)
        K = self.internal_k if node_type == 0 else self.istore_k
        if used > 2 * K or p + 24 + (2 * K + 1) * ksize + 2 * K * 8 > self.size:
            raise H5FormatError("B-tree node at %d: %d entries for K %d, or short" % (addr, used, K))
        q = p + 24
        out = []
        for i in range(used):
            key = q
            child = _u(b, q + ksize, 8)
            q += ksize + 8
            if level > 0:
                out.extend(self._btree_children(child, node_type, rank))
            elif node_type == 0:
                out.append(child)
            else:
                nbytes, mask = _u(b, key, 4), _u(b, key + 4, 4)
                offs = [_u(b, key + 8 + 8 * d, 8) for d in range(rank)]
                out.append((child, nbytes, mask, offs))
        return out

    # -- messages -----------------------------------------------------------
    def _dataspace(self, d, p):
        ver, rank, flags = d[p], d[p + 1], d[p + 2]
        if ver == 1:
            q = p + 8
            kind = 1 if rank > 0 else 0
        elif ver == 2:
            kind = d[p + 3]
            q = p + 4
        else:
            raise H5FormatError("dataspace version %d" % ver)
        dims = tuple(_u(d, q + 8 * i, 8) for i in range(rank))
        q += 8 * rank
        maxdims = None
        if flags & 1:
            maxdims = tuple(None if _u(d, q + 8 * i, 8) == UNDEF else _u(d, q + 8 * i, 8) for i in range(rank))
        if kind == 2:
            return None, None
        return dims, maxdims

    def _datatype(self, d, p):
        cv = d[p]
        cls, ver = cv & 0x0F, cv >> 4
        bits = d[p + 1] | (d[p + 2] << 8) | (d[p + 3] << 16)
        size = _u(d, p + 4, 4)
        if cls == 0:
            if bits & 1:
                raise H5FormatError("big-endian integer")
            return np.dtype(("<i%d" if bits & 0x08 else "<u%d") % size), 12
        if cls == 1:
            if bits & 1 or size not in (4, 8):
                raise H5FormatError("floating-point type of %d bytes" % size)
            return np.dtype("<f%d" % size), 20
        if cls == 3:
            return np.dtype("S%d" % size), 8
        raise H5FormatError("datatype class %d (version %d)" % (cls, ver))

    def _layout(self, d):
        ver = d[0]
        if ver != 3:
            raise H5FormatError("layout version %d" % ver)
        cls = d[1]
        if cls == 0:
            n = _u(d, 2, 2)
            return (0, d[4:4 + n])
        if cls == 1:
            return (1, _u(d, 2, 8), _u(d, 10, 8))
        if cls == 2:
            rank = d[2]
            addr = _u(d, 3, 8)
            dims = [_u(d, 11 + 4 * i, 4) for i in range(rank)]
            return (2, addr, dims[:-1], dims[-1])
        raise H5FormatError("layout class %d" % cls)

    def _filters(self, d):
        ver, n = d[0], d[1]
        out = []
        q = 8 if ver == 1 else 2
        for _ in range(n):
            fid = _u(d, q, 2)
            if ver == 1 or fid >= 256:
                nlen = _u(d, q + 2, 2)
                q += 4
            else:
                nlen = 0
                q += 2
            flags, nval = _u(d, q, 2), _u(d, q + 2, 2)
            q += 4
            q += ((nlen + 7) // 8) * 8 if ver == 1 else nlen
            vals = [_u(d, q + 4 * i, 4) for i in range(nval)]
            q += 4 * nval
            if ver == 1 and nval % 2:
                q += 4
            out.append((fid, flags, vals))
        return out

    def _attribute(self, d):
        ver = d[0]
        if ver == 1:
            nlen, tlen, slen = _u(d, 2, 2), _u(d, 4, 2), _u(d, 6, 2)
            pad = lambda n: (n + 7) // 8 * 8
            q = 8
            name = d[q:q + nlen].split(b"\0")[0].decode()
            q += pad(nlen)
            dt, _ = self._datatype(d, q)
            q += pad(tlen)
            dims, _ = self._dataspace(d, q)
            q += pad(slen)
        elif ver in (2, 3):
            nlen, tlen, slen = _u(d, 2, 2), _u(d, 4, 2), _u(d, 6, 2)
            q = 8 if ver == 2 else 9
            name = d[q:q + nlen].split(b"\0")[0].decode()
            q += nlen
            dt, _ = self._datatype(d, q)
            q += tlen
            dims, _ = self._dataspace(d, q)
            q += slen
        else:
            raise H5FormatError("attribute version %d" % ver)
        n = int(np.prod(dims)) if dims else 1
        val = np.frombuffer(d, dtype=dt, count=n, offset=q)
        if dims:
            val = val.reshape(dims)
        else:
            val = val[0]
        if dt.kind == "S" and n == 1:
            val = np.asarray(val).ravel()[0].split(b"\0")[0].decode()
        return name, val

    # -- raw data -----------------------------------------------------------
    def _read_dataset(self, ds):
        shape, dt = ds.shape, ds.dtype
        n = int(np.prod(shape)) if shape else 1
        lay = ds.layout
        if lay[0] == 0:
            return np.frombuffer(lay[1], dtype=dt, count=n).reshape(shape).copy()
        if lay[0] == 1:
            if lay[1] == UNDEF:
                return np.zeros(shape, dtype=dt)
            p = self._addr(lay[1])
            return np.frombuffer(self.b, dtype=dt, count=n, offset=p).reshape(shape).copy()
        _, btree, cdims, esize = lay
        if esize != dt.itemsize:
            raise H5FormatError("chunk element size %d for a %d-byte type" % (esize, dt.itemsize))
        out = np.zeros(shape, dtype=dt)
        rank = len(shape)
        for addr, nbytes, mask, offs in self._btree_children(btree, 1, rank):
            raw = bytes(self.b[self._addr(addr):self._addr(addr) + nbytes])
            for i in reversed(range(len(ds.filters))):
                fid, _, vals = ds.filters[i]
                if mask & (1 << i):
                    continue
                if fid == 1:
                    raw = zlib.decompress(raw)
                elif fid == 2:
                    es = vals[0] if vals else dt.itemsize
                    a = np.frombuffer(raw, dtype=np.uint8)
                    m = len(a) // es
                    raw = a[:m * es].reshape(es, m).T.tobytes() + a[m * es:].tobytes()
                elif fid == 3:
                    raw = raw[:-4]
                else:
                    raise H5FormatError("filter %d" % fid)
            chunk = np.frombuffer(raw, dtype=dt, count=int(np.prod(cdims))).reshape(cdims)
            dst = tuple(slice(o, min(o + c, s)) for o, c, s in zip(offs, cdims, shape))
            src = tuple(slice(0, sl.stop - sl.start) for sl in dst)
            out[dst] = chunk[src]
        return out


class LMFile:
    """A `.lm` file opened for reading, with the reference's SimulationFile
    accessors (io/SimulationFile.cpp) over the layout above."""

    def __init__(self, path):
        self.h5 = H5File(path)
        if self.h5.userblock[:4] != b"LMH5":
            self.h5.close()
            raise H5FormatError("%s is not a Lattice Microbes file (no LMH5 user block)" % path)
        self.version = int(np.asarray(self.h5.root.attrs["formatVersion"]).ravel()[0])

    def close(self):
        self.h5.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __getitem__(self, path):
        return self.h5[path]

    def parameters(self):
        """/Parameters as strings, as SimulationFile::parseParameter
        (io/SimulationFile.cpp:260-300) reads them: in format 2 the 8-byte
        floating-point attributes, printed with %e; from format 3 on the
        string attributes.  Other attributes are skipped."""
        out = {}
        for k, v in self.h5["Parameters"].attrs.items():
            a = np.asarray(v)
            if self.version == 2 and a.dtype == np.float64:
                out[k] = "%e" % float(a.ravel()[0])
            elif self.version >= 3 and isinstance(v, str):
                out[k] = v
        return out

    def _attr_uint(self, group, name):
        return int(np.asarray(self.h5[group].attrs[name]).ravel()[0])

    def reaction_model(self):
        """/Model/Reaction as SimulationFile::getReactionModel
        (io/SimulationFile.cpp:363-466) reads it: without a numberReactions
        attribute only the species count; otherwise the initial counts and,
        when there are reactions, per reaction its type, its rate constants up
        to the first NaN of the 10 columns and its noise (variance, tau) when
        both are positive, and the S and D matrices flattened (species major).
        Returns None when the file has no reaction model."""
        if "Model/Reaction" not in self.h5.root:
            return None
        g = self.h5["Model/Reaction"]
        ns = int(np.asarray(g.attrs["numberSpecies"]).ravel()[0])
        m = {"numberSpecies": ns, "numberReactions": 0, "initialSpeciesCounts": [], "reactions": [],
             "stoichiometricMatrix": [], "dependencyMatrix": []}
        if "numberReactions" not in g.attrs:
            return m
        init = g["InitialSpeciesCounts"].read()
        if init.shape != (ns,) or init.dtype.itemsize != 4:
            raise H5FormatError("InitialSpeciesCounts has shape %s" % (init.shape,))
        m["initialSpeciesCounts"] = [int(v) for v in init.astype(np.int64)]
        nr = int(np.asarray(g.attrs["numberReactions"]).ravel()[0])
        m["numberReactions"] = nr
        if nr == 0:
            return m
        types = g["ReactionTypes"].read()
        k = g["ReactionRateConstants"].read()
        S = g["StoichiometricMatrix"].read()
        D = g["DependencyMatrix"].read()
        if types.shape != (nr,) or k.shape != (nr, 10) or S.shape != (ns, nr) or D.shape != (ns, nr):
            raise H5FormatError("reaction tables of inconsistent shape")
        noise = g["ReactionRateNoise"].read() if "ReactionRateNoise" in g else None
        if noise is not None and noise.shape != (nr, 2):
            raise H5FormatError("ReactionRateNoise has shape %s" % (noise.shape,))
        for i in range(nr):
            rates = []
            for v in k[i]:
                if np.isnan(v):
                    break
                rates.append(float(v))
            r = {"type": int(types[i]), "rateConstants": rates, "noise": None}
            if noise is not None:
                nvar, ntau = float(noise[i, 0]), float(noise[i, 1])
                if nvar > 0.0 and ntau > 0.0:
                    r["noise"] = (nvar, ntau)
            m["reactions"].append(r)
        m["stoichiometricMatrix"] = [int(v) for v in S.astype(np.int64).ravel()]
        m["dependencyMatrix"] = [int(v) for v in D.astype(np.int64).ravel()]
        return m

    def diffusion_model(self):
        g = self.h5["Model/Diffusion"]
        m = {k: (v.item() if hasattr(v, "item") and np.size(v) == 1 else v) for k, v in g.attrs.items()}
        for name in ("DiffusionMatrix", "ReactionLocationMatrix", "Lattice", "LatticeSites"):
            if name in g:
                m[name] = g[name].read()
        return m

    def replicates(self):
        return sorted(int(k) for k in self.h5["Simulations"].keys())

    def _rep(self, replicate):
        return self.h5["Simulations/%07d" % replicate]

    def species_counts(self, replicate):
        g = self._rep(replicate)
        return g["SpeciesCountTimes"].read(), g["SpeciesCounts"].read()

    def lattice_times(self, replicate):
        g = self._rep(replicate)
        return g["LatticeTimes"].read() if "LatticeTimes" in g else np.zeros(0)

    def lattice(self, replicate, index):
        """Frame `index`, shape (X, Y, Z, particles per site)."""
        return self._rep(replicate)["Lattice/%010d" % index].read()

    def site_times(self, replicate):
        g = self._rep(replicate)
        return g["SiteTimes"].read() if "SiteTimes" in g else np.zeros(0)

    def sites(self, replicate, index):
        """Site-type frame `index`, shape (X, Y, Z)."""
        return self._rep(replicate)["Sites/%010d" % index].read()

    # The reference's SimulationFile getter names (io/SimulationFile.h:134-266).
    def getParameters(self):
        return self.parameters()

    def getParameter(self, key, defaultValue=""):
        return self.parameters().get(key, defaultValue)

    def getReactionModel(self):
        return self.reaction_model()

    def getDiffusionModel(self):
        return self.diffusion_model()

    def getLatticeTimes(self, replicate):
        return list(self.lattice_times(replicate))

    def getLattice(self, replicate, latticeIndex):
        return self.lattice(replicate, latticeIndex)

    def getSpeciesCountTimes(self, replicate):
        return list(self.species_counts(replicate)[0])

    def getSpeciesCounts(self, replicate):
        """{time: counts of species 1..ns} as SimulationFile::getSpeciesCounts."""
        t, c = self.species_counts(replicate)
        return {float(a): [int(v) for v in b] for a, b in zip(t, c)}

    def max_counts(self, replicate):
        g = self._rep(replicate)
        if "MaxParticleCounts" not in g:
            return None
        return g["MaxParticleCounts"].read(), g["MaxSiteCounts"].read()


class LMFileWriter:
    """A new `.lm` file written through lmb_lmfile_* (include/lmb_lmfile.h):
    the reference's SimulationFile create / setParameter / setReactionModel /
    setDiffusionModel / setDiffusionModelLattice and the trajectory records
    its DataOutputQueue writes.  Lattice frames go through a writer thread;
    `flush` makes the file on disk complete, `close` flushes and closes."""

    def __init__(self, path):
        import ctypes as C
        from . import _lib as L
        self._C, self._L = C, L
        h = L.vp()
        L.check(L.lib().lmb_lmfile_create(os.fsencode(path), C.byref(h)), "lmb_lmfile_create(%s)" % path)
        self.h = h
        self.path = path
        self.checkpoint_path = None  # where checkpoint() puts the copy (None: "<path>.chk")

    def _p(self, a, t):
        return a.ctypes.data_as(self._C.POINTER(t)) if a is not None else None

    def set_parameter(self, key, value):
        self._L.check(self._L.lib().lmb_lmfile_set_parameter(self.h, key.encode(), str(value).encode()))

    def set_reaction_model(self, initial_counts, types, rate_constants, S, D, noise=None):
        """rate_constants [nr][<=10] (padded with NaN), S and D [ns][nr],
        noise [nr][2] or None."""
        C, L = self._C, self._L
        init = np.ascontiguousarray(initial_counts, np.uint32)
        ns = init.size
        types = np.ascontiguousarray(types, np.uint32)
        nr = types.size
        k = np.full((nr, 10), np.nan)
        for i, row in enumerate(rate_constants):
            row = np.asarray(row, np.float64).ravel()
            k[i, :row.size] = row
        S = np.ascontiguousarray(np.asarray(S).reshape(ns, nr), np.int32)
        D = np.ascontiguousarray(np.asarray(D).reshape(ns, nr), np.uint32)
        nz = None if noise is None else np.ascontiguousarray(np.asarray(noise).reshape(nr, 2), np.float64)
        L.check(L.lib().lmb_lmfile_set_reaction_model(self.h, ns, nr, self._p(init, C.c_uint32),
                                                      self._p(types, C.c_uint32), self._p(k, C.c_double),
                                                      self._p(nz, C.c_double), self._p(S, C.c_int32),
                                                      self._p(D, C.c_uint32)))

    def set_diffusion_model(self, spacing, X, Y, Z, particles_per_site, bytes_per_particle, DF, RL):
        """DF [nst][nst][ns], RL [nr][nst]."""
        C, L = self._C, self._L
        DF = np.ascontiguousarray(DF, np.float64)
        nst, ns = DF.shape[0], DF.shape[2]
        RL = np.ascontiguousarray(np.asarray(RL).reshape(-1, nst), np.uint32)
        nr = RL.shape[0]
        L.check(L.lib().lmb_lmfile_set_diffusion_model(self.h, ns, nr, nst, float(spacing), X, Y, Z,
                                                       particles_per_site, bytes_per_particle,
                                                       self._p(DF, C.c_double), self._p(RL, C.c_uint32)))

    def set_diffusion_model_lattice(self, particles, sites):
        """Row-major particles [X][Y][Z][P] (uint8 or uint32) and sites [X][Y][Z]."""
        C, L = self._C, self._L
        particles = np.ascontiguousarray(particles)
        sites = np.ascontiguousarray(sites, np.uint8)
        L.check(L.lib().lmb_lmfile_set_diffusion_model_lattice(self.h, particles.ctypes.data,
                                                               self._p(sites, C.c_uint8)))

    def append_species_counts(self, replicate, times, counts):
        C, L = self._C, self._L
        times = np.ascontiguousarray(times, np.float64).ravel()
        counts = np.ascontiguousarray(counts, np.int32)
        counts = counts.reshape(times.size, counts.shape[-1] if counts.ndim == 2 else -1)
        L.check(L.lib().lmb_lmfile_append_species_counts(self.h, replicate, times.size, counts.shape[1],
                                                         self._p(times, C.c_double), self._p(counts, C.c_int32)))

    def append_lattice(self, replicate, time, particles):
        """A host frame [X][Y][Z][P], uint8 (ByteLattice) or uint32 (IntLattice)."""
        particles = np.ascontiguousarray(particles)
        X, Y, Z, P = particles.shape
        bpp = particles.dtype.itemsize
        self._L.check(self._L.lib().lmb_lmfile_append_lattice(self.h, replicate, float(time), X, Y, Z, P, bpp,
                                                              particles.ctypes.data))

    def append_lattice_device(self, replicate, time, lattice):
        """The current state of a solver.Lattice on the device, asynchronously."""
        self._L.check(self._L.lib().lmb_lmfile_append_lattice_device(self.h, replicate, float(time), lattice.handle))

    def append_sites(self, replicate, time, sites):
        sites = np.ascontiguousarray(sites, np.uint8)
        X, Y, Z = sites.shape
        self._L.check(self._L.lib().lmb_lmfile_append_sites(self.h, replicate, float(time), X, Y, Z,
                                                            self._p(sites, self._C.c_uint8)))

    def append_sites_device(self, replicate, time, lattice):
        self._L.check(self._L.lib().lmb_lmfile_append_sites_device(self.h, replicate, float(time), lattice.handle))

    def write_max_counts(self, replicate, max_particle_counts, max_site_counts):
        C = self._C
        mp = np.ascontiguousarray(max_particle_counts, np.uint32)
        ms = np.ascontiguousarray(max_site_counts, np.uint32)
        self._L.check(self._L.lib().lmb_lmfile_write_max_counts(self.h, replicate, self._p(mp, C.c_uint32), mp.size,
                                                                self._p(ms, C.c_uint32), ms.size))

    # -- generic objects (carrying an existing file's contents over) ----------
    _CODES = {np.dtype("u1"): 1, np.dtype("i1"): 2, np.dtype("<u2"): 3, np.dtype("<i2"): 4, np.dtype("<u4"): 5,
              np.dtype("<i4"): 6, np.dtype("<u8"): 7, np.dtype("<i8"): 8, np.dtype("<f4"): 9, np.dtype("<f8"): 10}

    def create_group(self, path):
        self._L.check(self._L.lib().lmb_lmfile_create_group(self.h, path.encode()))

    def set_attribute(self, path, name, value):
        """A string (scalar), or a numeric array / number (rank as given;
        a Python number becomes a one-element array)."""
        C, L = self._C, self._L
        if isinstance(value, (str, bytes)):
            v = value.encode() if isinstance(value, str) else value
            buf = np.frombuffer(v + b"\0", dtype=np.uint8).copy()
            L.check(L.lib().lmb_lmfile_set_attribute(self.h, path.encode(), name.encode(), 11, 0, None,
                                                     buf.ctypes.data, buf.size))
            return
        a = np.asarray(value)
        if a.dtype.kind == "S":
            a = np.ascontiguousarray(a)
            dims = np.asarray(a.shape, dtype=np.uint64)
            L.check(L.lib().lmb_lmfile_set_attribute(self.h, path.encode(), name.encode(), 11, a.ndim,
                                                     self._p(dims, C.c_uint64), a.ctypes.data, a.dtype.itemsize))
            return
        if a.ndim == 0:
            a = a.reshape(1)
        a = np.ascontiguousarray(a, dtype=a.dtype.newbyteorder("<"))
        code = self._CODES.get(a.dtype)
        if code is None:
            raise TypeError("attribute type %s" % a.dtype)
        dims = np.asarray(a.shape, dtype=np.uint64)
        L.check(L.lib().lmb_lmfile_set_attribute(self.h, path.encode(), name.encode(), code, a.ndim,
                                                 self._p(dims, C.c_uint64), a.ctypes.data, 0))

    def write_dataset(self, group, name, data, chunks=None, gzip=-1, extendable=False):
        C, L = self._C, self._L
        a = np.ascontiguousarray(data)
        a = np.ascontiguousarray(a, dtype=a.dtype.newbyteorder("<"))
        code = self._CODES.get(a.dtype)
        if code is None:
            raise TypeError("dataset type %s" % a.dtype)
        dims = np.asarray(a.shape, dtype=np.uint64)
        cd = None if chunks is None else np.asarray(chunks, dtype=np.uint64)
        L.check(L.lib().lmb_lmfile_write_dataset(self.h, group.encode(), name.encode(), code, a.ndim,
                                                 self._p(dims, C.c_uint64), self._p(cd, C.c_uint64), int(gzip),
                                                 int(bool(extendable)), a.ctypes.data if a.size else None))

    def copy_from(self, src):
        """Every group, attribute and dataset of an open H5File (or LMFile),
        with each dataset's chunking, gzip level and extendability."""
        h5 = src.h5 if isinstance(src, LMFile) else src

        def walk(g, path):
            if path:
                self.create_group(path)
            for k, v in g.attrs.items():
                self.set_attribute(path or "/", k, v)
            for name in g.keys():
                o = g[name]
                sub = path + "/" + name if path else name
                if isinstance(o, Group):
                    walk(o, sub)
                    continue
                gz = -1
                for fid, _, vals in o.filters:
                    if fid == 1:
                        gz = vals[0] if vals else 6
                ext = o.maxshape is not None and len(o.maxshape) > 0 and o.maxshape[0] is None
                self.write_dataset(path or "/", name, o.read(), chunks=o.chunks, gzip=gz, extendable=ext)
                for k, v in o.attrs.items():
                    self.set_attribute(sub, k, v)

        walk(h5.root, "")

    def flush(self):
        self._L.check(self._L.lib().lmb_lmfile_flush(self.h))

    def checkpoint(self):
        """SimulationFile::checkpoint: the file so far, complete, copied to
        "<path>.chk"; returns that name."""
        buf = self._C.create_string_buffer(len(os.fsencode(self.path)) + 16)
        self._L.check(self._L.lib().lmb_lmfile_checkpoint(self.h, buf, len(buf)))
        chk = os.fsdecode(buf.value)
        if self.checkpoint_path:
            os.replace(chk, self.checkpoint_path)
            chk = self.checkpoint_path
        return chk

    def stats(self):
        C = self._C
        frames, nbytes = C.c_uint64(), C.c_uint64()
        self._L.check(self._L.lib().lmb_lmfile_stats(self.h, C.byref(frames), C.byref(nbytes)))
        return frames.value, nbytes.value

    def close(self):
        if self.h:
            h, self.h = self.h, None
            self._L.check(self._L.lib().lmb_lmfile_close(h))

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
