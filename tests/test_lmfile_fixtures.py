"""The `.lm` reader against the HDF5 files the reference's own tests read
(testing/data/lm/io/hdf5/*.h5, written by libhdf5 and Matlab), with the values
testing/c/lm/io/hdf5/simulation_file.cpp expects of them.  The fixtures are
committed under tests/golden/lmfile/ (copied byte for byte by
tests/golden/make_lmfile_fixtures.py)."""
import os

import numpy as np
import pytest

from lattice_microbes_b200.lmfile import H5FormatError, LMFile

D = os.path.join(os.path.dirname(__file__), "golden", "lmfile")


def path(name):
    return os.path.join(D, name)


def test_not_an_hdf5_file():
    """OpenNonHDF5File (simulation_file.cpp:82-89): a 5-byte text file."""
    with pytest.raises(H5FormatError):
        LMFile(path("SimulationFile_1.h5"))


def test_parameters_format_2():
    """GetParameterV2 (simulation_file.cpp:119-128): doubles, strings ignored."""
    with LMFile(path("SimulationFile_2.h5")) as f:
        assert f.version == 2
        p = f.parameters()
        assert "unused1" not in p
        assert float(p["test1"]) == pytest.approx(2.3, rel=1e-4)
        assert float(p["test2"]) == pytest.approx(5.7e-16, rel=1e-4)
        assert "test3" not in p


def test_parameters_format_3():
    """GetParameterV3 (simulation_file.cpp:130-141): strings; the integer
    attribute test4 is not a parameter."""
    with LMFile(path("SimulationFile_3.h5")) as f:
        assert f.version == 3
        p = f.parameters()
        assert float(p["test1"]) == pytest.approx(2.3, rel=1e-4)
        assert float(p["test2"]) == pytest.approx(5.7e-16, rel=1e-4)
        assert p["test3"] == "testing"
        assert p.get("test4", "") == ""


def test_reaction_model_without_reaction_count():
    """simulation_file.cpp:505-513."""
    with LMFile(path("SimulationFile_GetReactionModel_NoReactionCount.h5")) as f:
        m = f.reaction_model()
        assert (m["numberSpecies"], m["numberReactions"], len(m["initialSpeciesCounts"])) == (5, 0, 0)


S57 = [1, -1, 0, -1, 0, 1, -1,
       -1, 1, 0, 0, 1, 1, -1,
       0, 0, 1, 1, 1, 1, -1,
       0, 0, -1, 0, 0, 1, -1,
       0, 0, 0, -1, 0, 1, -1]
D57 = [1, 0, 0, 1, 0, 0, 1,
       0, 1, 0, 1, 0, 0, 1,
       0, 0, 1, 0, 1, 0, 1,
       0, 1, 0, 0, 1, 1, 1,
       1, 0, 0, 0, 0, 1, 0]
RATES = [[1.5], [7.0], [16.7, 17.3], [1678.0, 1.0e12], [2.0, 3.0, 4.0, 5.0, 6.0, 7.0, 8.0, 9.0, 10.0, 11.0],
         [5.6], [6.7]]


@pytest.mark.parametrize("name", ["SimulationFile_GetReactionModel.h5", "SimulationFile_GetReactionModel_Noise.h5"])
def test_reaction_model(name):
    """simulation_file.cpp:515-584 and 586-666."""
    with LMFile(path(name)) as f:
        m = f.reaction_model()
    assert (m["numberSpecies"], m["numberReactions"]) == (5, 7)
    assert m["initialSpeciesCounts"] == [11, 13, 17, 19, 23]
    assert [r["type"] for r in m["reactions"]] == [1, 1, 2, 2, 91, 98, 99]
    for r, want in zip(m["reactions"], RATES):
        assert r["rateConstants"] == pytest.approx(want, rel=1e-11)
    assert m["stoichiometricMatrix"] == S57
    assert m["dependencyMatrix"] == D57
    noise = [r["noise"] for r in m["reactions"]]
    if "Noise" in name:
        assert [n is not None for n in noise] == [False, True, False, False, True, True, False]
        assert noise[1] == pytest.approx((11.11, 1e5), rel=1e-11)
        assert noise[4] == pytest.approx((4.4, 1e14), rel=1e-11)
        assert noise[5] == pytest.approx((5.555, 1e15), rel=1e-11)
    else:
        assert noise == [None] * 7


def test_diffusion_model_and_lattice():
    """GetDiffusionModel / GetDiffusionModelLattice (simulation_file.cpp:
    1058-1200): the sizes, and the Matlab-written lattice read in file order
    as l[x + y X + z X Y + p X Y Z] = 20 p + 50 z + X y + x, sites + 1."""
    with LMFile(path("SimulationFile_GetDiffusionModel.h5")) as f:
        d = f.diffusion_model()
    assert d["latticeSpacing"] == 16.0
    X, Y, Z, P = d["latticeXSize"], d["latticeYSize"], d["latticeZSize"], d["particlesPerSite"]
    assert (X, Y, Z, P) == (3, 4, 5, 2)
    l1 = d["Lattice"].ravel()
    l2 = d["LatticeSites"].ravel()
    for p in range(P):
        for z in range(Z):
            for y in range(Y):
                for x in range(X):
                    assert l1[x + y * X + z * X * Y + p * X * Y * Z] == p * 20 + z * 50 + y * X + x
    for z in range(Z):
        for y in range(Y):
            for x in range(X):
                assert l2[x + y * X + z * X * Y] == z * 50 + y * X + x + 1


def test_spatial_model_spheres_chunked():
    """GetSpatialModelObjects (simulation_file.cpp:1176-1200): 382 spheres in
    an extendable dataset of 100-row chunks that libhdf5 indexed with a chunk
    B-tree, and the empty extendable SpeciesCounts / SpeciesCountTimes the
    reference's createReplicateHandles makes."""
    with LMFile(path("SimulationFile_GetSpatialModelObjects.h5")) as f:
        ds = f["Simulations/0000001/Model/Spatial/Spheres"]
        assert ds.chunks == (100, 5) and ds.maxshape == (None, 5)
        s = ds.read()
        sc = f["Simulations/0000000/SpeciesCounts"]
        assert sc.shape == (0, 1) and sc.maxshape == (None, 1) and sc.chunks == (100, 1)
        assert sc.read().shape == (0, 1) and sc.dtype == np.int32
    assert s.shape == (382, 5)
    for i, (xc, yc, zc, r, t) in ((0, (239.6, 155.9, 143.6, 10.4, 21.0)), (100, (333.0, 279.8, 719.6, 4.0, 25.0)),
                                  (381, (76.7, 191.7, 949.0, 1.7, 32.0))):
        assert s[i, :3] == pytest.approx([xc, yc, zc], rel=1e-3)
        assert (s[i, 3], s[i, 4]) == pytest.approx((r, t), rel=1e-11)


def _messages(f, path):
    parts = path.split("/")
    node = f.h5.root
    for p in parts[:-1]:
        node = node[p]
    return {t: d for t, d in f.h5._messages(node._entries()[parts[-1]])}


def test_writer_encodes_the_replicate_datasets_as_libhdf5(tmp_path):
    """The dataspace, datatype, fill-value and layout messages the writer
    gives a new replicate's SpeciesCounts (i32, 100 x 1 chunks, unlimited
    rows) and SpeciesCountTimes are byte for byte the ones libhdf5 wrote for
    the reference's createReplicateHandles in the fixture."""
    from lattice_microbes_b200.lmfile import LMFileWriter
    p = str(tmp_path / "r.lm")
    with LMFileWriter(p) as w:
        w.append_species_counts(0, np.zeros(0), np.zeros((0, 1), np.int32))
    with LMFile(path("SimulationFile_GetSpatialModelObjects.h5")) as ref, LMFile(p) as got:
        for name in ("SpeciesCounts", "SpeciesCountTimes"):
            a = _messages(ref, "Simulations/0000000/" + name)
            b = _messages(got, "Simulations/0000000/" + name)
            for t in (0x0001, 0x0003, 0x0005, 0x0008):
                assert a[t] == b[t], (name, hex(t), a[t].hex(), b[t].hex())


def test_writer_encodes_uint_attributes_as_libhdf5(tmp_path):
    """The root's formatVersion attribute (H5LTset_attribute_uint): the same
    name, datatype and dataspace encoding as libhdf5's in the fixture, with
    this file's version 4 in place of the fixture's 2."""
    from lattice_microbes_b200.lmfile import LMFileWriter
    p = str(tmp_path / "a.lm")
    LMFileWriter(p).close()
    with LMFile(path("SimulationFile_2.h5")) as ref, LMFile(p) as got:
        a = [d for t, d in ref.h5._messages(ref.h5.root_addr) if t == 0x000C]
        b = [d for t, d in got.h5._messages(got.h5.root_addr) if t == 0x000C]
        assert len(a) == len(b) == 1
        assert a[0][:56] == b[0][:56] and a[0][56:60] == (2).to_bytes(4, "little")
        assert b[0][56:60] == (4).to_bytes(4, "little")
        assert got.version == 4
