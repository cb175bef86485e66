"""The `.lm` writer (include/lmb_lmfile.h) on the CPU through its host-buffer
calls: every record written comes back through the reader, which the
libhdf5-written fixtures pin (tests/test_lmfile_fixtures.py); the HDF5
structures are checked against the forms libhdf5 writes (user block,
superblock fields, full-size B-tree nodes, multi-level B-trees for groups of
more than 256 entries and datasets of more than 64 chunks)."""
import os

import numpy as np
import pytest

from lattice_microbes_b200.lmfile import LMFile, LMFileWriter


def _model(w, rng, ns=5, nr=7, nst=3):
    init = rng.integers(0, 100, ns)
    types = rng.integers(0, 4, nr)
    k = [rng.uniform(0.1, 10.0, 1 + (i % 3)) for i in range(nr)]
    S = rng.integers(-1, 2, (ns, nr))
    D = rng.integers(0, 2, (ns, nr))
    noise = np.zeros((nr, 2))
    noise[1] = (11.11, 1e5)
    w.set_reaction_model(init, types, k, S, D, noise=noise)
    return init, types, k, S, D, noise


def test_round_trip(tmp_path):
    rng = np.random.default_rng(5)
    p = str(tmp_path / "t.lm")
    X, Y, Z, P, ns, nst = 20, 18, 35, 8, 5, 3
    with LMFileWriter(p) as w:
        w.set_parameter("timestep", "5e-05")
        w.set_parameter("maxTime", "1.0")
        w.set_parameter("timestep", "2.5e-05")  # replaced, as setParameter does
        init, types, k, S, D, noise = _model(w, rng, ns=ns)
        DF = rng.uniform(0, 1, (nst, nst, ns))
        RL = rng.integers(0, 2, (7, nst))
        w.set_diffusion_model(16e-9, X, Y, Z, P, 1, DF, RL)
        lat0 = rng.integers(0, ns + 1, (X, Y, Z, P)).astype(np.uint8)
        sites0 = rng.integers(0, nst, (X, Y, Z)).astype(np.uint8)
        w.set_diffusion_model_lattice(lat0, sites0)
        frames = [rng.integers(0, 6, (X, Y, Z, P)).astype(np.uint8) * (rng.random((X, Y, Z, P)) < 0.1)
                  for _ in range(3)]
        for i, fr in enumerate(frames):
            w.append_lattice(1, 0.5 * i, fr)
        times = np.arange(250) * 0.01
        counts = rng.integers(0, 1000, (250, ns))
        w.append_species_counts(1, times[:120], counts[:120])
        w.append_species_counts(1, times[120:], counts[120:])
        w.append_sites(1, 0.0, sites0)
        w.append_sites(1, 1.0, (sites0 + 1) % nst)
        w.write_max_counts(1, np.arange(ns + 1), np.array([0, 7, 9]))
        ints = rng.integers(0, 2 ** 32, (9, 7, 5, 4), dtype=np.uint64).astype(np.uint32)
        w.append_lattice(2, 0.0, ints)
        w.flush()
        assert w.stats()[0] == 6
    with open(p, "rb") as fh:
        head = fh.read(1024)
    assert head[:4] == b"LMH5" and head[512:520] == b"\x89HDF\r\n\x1a\n"
    assert int.from_bytes(head[512 + 24:512 + 32], "little") == 512      # base address
    assert int.from_bytes(head[512 + 40:512 + 48], "little") == os.path.getsize(p)  # absolute EOF
    with LMFile(p) as f:
        assert f.version == 4
        assert f.parameters() == {"timestep": "2.5e-05", "maxTime": "1.0"}
        m = f.reaction_model()
        assert m["initialSpeciesCounts"] == [int(v) for v in init]
        assert [r["type"] for r in m["reactions"]] == [int(t) for t in types]
        for r, want in zip(m["reactions"], k):
            assert r["rateConstants"] == list(want)
        assert m["reactions"][1]["noise"] == (11.11, 1e5)
        assert m["reactions"][0]["noise"] is None
        assert m["stoichiometricMatrix"] == [int(v) for v in S.ravel()]
        d = f.diffusion_model()
        assert (d["latticeXSize"], d["latticeYSize"], d["latticeZSize"], d["particlesPerSite"]) == (X, Y, Z, P)
        assert d["latticeSpacing"] == 16e-9 and d["numberSiteTypes"] == nst and d["bytes_per_particle"] == 1
        assert np.array_equal(d["DiffusionMatrix"], DF) and np.array_equal(d["ReactionLocationMatrix"], RL)
        assert np.array_equal(d["Lattice"], lat0) and np.array_equal(d["LatticeSites"], sites0)
        assert f.h5["Model/Diffusion/Lattice"].chunks == (16, 16, 16, P)
        assert f.replicates() == [1, 2]
        t, c = f.species_counts(1)
        assert np.array_equal(t, times) and np.array_equal(c, counts)
        sc = f.h5["Simulations/0000001/SpeciesCounts"]
        assert sc.dtype == np.int32 and sc.maxshape == (None, ns) and sc.chunks == (100, ns)
        assert np.array_equal(f.lattice_times(1), [0.0, 0.5, 1.0])
        for i, fr in enumerate(frames):
            got = f.lattice(1, i)
            assert got.dtype == np.uint8 and np.array_equal(got, fr)
        assert np.array_equal(f.sites(1, 1), (sites0 + 1) % nst)
        assert np.array_equal(f.site_times(1), [0.0, 1.0])
        mp, ms = f.max_counts(1)
        assert np.array_equal(mp, np.arange(ns + 1)) and np.array_equal(ms, [0, 7, 9])
        got = f.lattice(2, 0)
        assert got.dtype == np.uint32 and np.array_equal(got, ints)
        assert f.species_counts(2)[1].shape == (0, ns)


def test_many_frames_and_chunks(tmp_path):
    """A group of 300 frames (38 symbol-table nodes: a two-level group B-tree)
    and a frame of 5 x 5 x 3 = 75 chunks (a two-level chunk B-tree)."""
    rng = np.random.default_rng(7)
    p = str(tmp_path / "m.lm")
    small = [rng.integers(0, 3, (2, 3, 4, 4)).astype(np.uint8) for _ in range(300)]
    big = rng.integers(0, 3, (80, 80, 48, 4)).astype(np.uint8)
    with LMFileWriter(p) as w:
        for i, fr in enumerate(small):
            w.append_lattice(0, float(i), fr)
        w.append_lattice(3, 0.0, big)
    with LMFile(p) as f:
        g = f.h5["Simulations/0000000/Lattice"]
        assert len(g.keys()) == 300
        for i in (0, 1, 137, 299):
            assert np.array_equal(f.lattice(0, i), small[i])
        assert np.array_equal(f.lattice_times(0), np.arange(300.0))
        assert np.array_equal(f.lattice(3, 0), big)


def test_flush_leaves_a_complete_file(tmp_path):
    """After flush the file is readable while it stays open for more frames."""
    p = str(tmp_path / "f.lm")
    a = np.ones((4, 4, 4, 8), np.uint8)
    w = LMFileWriter(p)
    w.append_lattice(0, 0.0, a)
    w.flush()
    with LMFile(p) as f:
        assert np.array_equal(f.lattice(0, 0), a)
    w.append_lattice(0, 1.0, 2 * a)
    w.close()
    with LMFile(p) as f:
        assert np.array_equal(f.lattice(0, 1), 2 * a) and np.array_equal(f.lattice_times(0), [0.0, 1.0])


def test_refuses_existing_file_and_bad_arguments(tmp_path):
    from lattice_microbes_b200 import _lib as L
    p = str(tmp_path / "e.lm")
    open(p, "w").close()
    with pytest.raises(L.LmbError) as e:
        LMFileWriter(p)
    assert e.value.status == L.LMB_E_IO
    with LMFileWriter(str(tmp_path / "g.lm")) as w:
        with pytest.raises(L.LmbError):
            w.write_max_counts(0, np.zeros(0), np.zeros(3))
        w.write_max_counts(0, np.zeros(3), np.zeros(3))
        with pytest.raises(L.LmbError):  # each written once
            w.write_max_counts(0, np.zeros(3), np.zeros(3))
        with pytest.raises(L.LmbError):  # no diffusion model yet
            w.set_diffusion_model_lattice(np.zeros((2, 2, 2, 8), np.uint8), np.zeros((2, 2, 2), np.uint8))


@pytest.mark.parametrize("name", ["SimulationFile_GetSpatialModelObjects.h5", "SimulationFile_GetReactionModel_Noise.h5",
                                  "SimulationFile_GetDiffusionModel.h5", "SimulationFile_3.h5"])
def test_copy_of_a_libhdf5_file(tmp_path, name):
    """Every group, attribute and dataset of a libhdf5-written file survives
    a copy through the writer (the runSolver path), with chunking and
    extendability; appends then extend the copied extendable datasets."""
    from lattice_microbes_b200.lmfile import Group
    src = os.path.join(os.path.dirname(__file__), "golden", "lmfile", name)
    p = str(tmp_path / "c.lm")
    with LMFile(src) as a, LMFileWriter(p) as w:
        w.copy_from(a)
    with LMFile(src) as a, LMFile(p) as b:
        assert a.version == b.version

        def same(ga, gb):
            assert sorted(ga.keys()) == sorted(gb.keys())
            assert sorted(ga.attrs) == sorted(gb.attrs)
            for k in ga.attrs:
                va, vb = ga.attrs[k], gb.attrs[k]
                assert (va == vb) if isinstance(va, str) else np.array_equal(va, vb)
            for k in ga.keys():
                oa, ob = ga[k], gb[k]
                if isinstance(oa, Group):
                    same(oa, ob)
                else:
                    assert oa.dtype == ob.dtype and oa.shape == ob.shape
                    assert (oa.maxshape or oa.shape) == (ob.maxshape or ob.shape)  # no max: fixed
                    assert oa.chunks == ob.chunks
                    assert oa.read().tobytes() == ob.read().tobytes()  # bit for bit (NaN included)
        same(a.h5.root, b.h5.root)
    if "Spatial" in name:
        p2 = str(tmp_path / "d.lm")
        with LMFile(p) as a, LMFileWriter(p2) as w:
            w.copy_from(a)
            w.append_species_counts(0, [0.5, 1.0], [[3], [4]])
        with LMFile(p2) as b:
            t, c = b.species_counts(0)
            assert np.array_equal(t, [0.5, 1.0]) and np.array_equal(c, [[3], [4]])


def test_gzip_chunks_are_zlib_level_1(tmp_path):
    """Each stored chunk is exactly zlib's level-1 stream of the chunk's
    bytes, as libhdf5's deflate filter (compress2) stores it."""
    import zlib
    rng = np.random.default_rng(3)
    a = (rng.random((20, 16, 16, 8)) < 0.02).astype(np.uint8) * 3
    p = str(tmp_path / "z.lm")
    with LMFileWriter(p) as w:
        w.write_dataset("g", "d", a, chunks=(16, 16, 16, 8), gzip=1)
    with LMFile(p) as f:
        ds = f.h5["g/d"]
        kids = f.h5._btree_children(ds.layout[1], 1, 4)
        assert len(kids) == 2
        for addr, nbytes, mask, offs in kids:
            chunk = np.zeros((16, 16, 16, 8), np.uint8)
            part = a[offs[0]:offs[0] + 16]
            chunk[:part.shape[0]] = part
            raw = bytes(f.h5.b[f.h5._addr(addr):f.h5._addr(addr) + nbytes])
            assert mask == 0 and raw == zlib.compress(chunk.tobytes(), 1)


def test_checkpoint_copies_the_file_so_far(tmp_path):
    """SimulationFile::checkpoint: the checkpoint is a complete file with the
    records written so far; the run goes on in the original."""
    p = str(tmp_path / "k.lm")
    a = np.arange(4 * 4 * 4 * 8, dtype=np.uint8).reshape(4, 4, 4, 8)
    w = LMFileWriter(p)
    w.set_parameter("maxTime", "2.0")
    w.append_lattice(1, 0.0, a)
    w.append_species_counts(1, [0.0], [[5, 6]])
    chk = w.checkpoint()
    assert chk == p + ".chk"
    w.append_lattice(1, 1.0, a + 1)
    w.close()
    with LMFile(chk) as f:
        assert f.getParameter("maxTime") == "2.0" and f.getParameter("absent", "x") == "x"
        assert f.getLatticeTimes(1) == [0.0] and np.array_equal(f.getLattice(1, 0), a)
        assert f.getSpeciesCounts(1) == {0.0: [5, 6]}
    with LMFile(p) as f:
        assert f.getLatticeTimes(1) == [0.0, 1.0] and np.array_equal(f.getLattice(1, 1), a + 1)


def test_oversized_attribute_is_refused(tmp_path):
    """A header message holds at most 64 KiB: a longer parameter is refused,
    and the file stays valid."""
    from lattice_microbes_b200 import _lib as L
    p = str(tmp_path / "big_attr.lm")
    with LMFileWriter(p) as w:
        with pytest.raises(L.LmbError) as e:
            w.set_parameter("long", "x" * 70000)
        assert e.value.status == L.LMB_E_ARG
        w.set_parameter("short", "y" * 60000)
    with LMFile(p) as f:
        assert f.parameters() == {"short": "y" * 60000}


def test_repeated_flushes_grow_the_file_linearly(tmp_path):
    """Flushes and checkpoints re-append only what changed: chunks of species
    count rows that were full at an earlier flush stay where they are, and
    groups no record touched keep their headers.  K flushes over R records
    add at most about one row chunk and a fixed amount of metadata per flush
    to the size a single flush gives, independent of R."""
    rng = np.random.default_rng(3)
    ns, R, every = 50, 2000, 10
    times = np.arange(R) * 0.5
    counts = rng.integers(0, 1000, (R, ns))
    one = str(tmp_path / "one.lm")
    with LMFileWriter(one) as w:
        w.append_lattice(1, 0.0, np.ones((8, 8, 8, 8), np.uint8))
        w.append_species_counts(1, times, counts)
        w.flush()
    many = str(tmp_path / "many.lm")
    K = 0
    with LMFileWriter(many) as w:
        w.append_lattice(1, 0.0, np.ones((8, 8, 8, 8), np.uint8))
        for r0 in range(0, R, every):
            w.append_species_counts(1, times[r0:r0 + every], counts[r0:r0 + every])
            if (r0 // every) % 50 == 49:
                w.checkpoint()
            else:
                w.flush()
            K += 1
    row_chunk = 100 * (4 * ns + 8)
    grown = os.path.getsize(many) - os.path.getsize(one)
    assert grown <= K * (row_chunk + 24 * 1024), (grown, K)
    with LMFile(many) as f:
        t, c = f.species_counts(1)
        assert np.array_equal(t, times) and np.array_equal(c, counts)
    with LMFile(many + ".chk") as f:
        t, c = f.species_counts(1)
        assert np.array_equal(t, times[:len(t)]) and len(t) == 2000
