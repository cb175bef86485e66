"""The `lm` module surface jLM and pyLM scripts use (lattice_microbes_b200.lm):
importing it makes `import lm` work; a model built through the protobuf-style
messages in jLM's order (jlm/jLM/LmInteract.py:55-84) is written by
SimulationFile and reads back unchanged; lm.simulationFile(name).setParameter
then close (jlm/jLM/RDME.py:450-453) changes that parameter and keeps the
rest of the file."""
import numpy as np

from lattice_microbes_b200 import configs


def _jlm_model(lm, spec, pps):
    """ReactionModel / DiffusionModel / lattice filled with jLM's calls."""
    rm = lm.ReactionModel()
    rm.set_number_reactions(spec.nr)
    rm.set_number_species(spec.ns)
    init = configs.species_counts(spec.lattice, spec.nsites, spec.slots, spec.bytes_per_slot, spec.ns)[1:]
    for c in init:
        rm.add_initial_species_count(int(c))
    for r in range(spec.nr):
        rm.add_reaction()
        rm.mutable_reaction(r).set_type(int(spec.rtype[r]))
        rm.mutable_reaction(r).add_rate_constant(float(np.ravel(spec.K)[r]))
    S = np.asarray(spec.S).reshape(spec.ns, spec.nr)
    D = np.asarray(spec.D).reshape(spec.ns, spec.nr)
    for s in range(spec.ns):
        for r in range(spec.nr):
            rm.add_stoichiometric_matrix(int(S[s, r]))
    for s in range(spec.ns):
        for r in range(spec.nr):
            rm.add_dependency_matrix(int(D[s, r]))
    dm = lm.DiffusionModel()
    dm.set_number_reactions(spec.nr)
    dm.set_number_species(spec.ns)
    dm.set_number_site_types(spec.nst)
    dm.set_lattice_x_size(spec.X)
    dm.set_lattice_y_size(spec.Y)
    dm.set_lattice_z_size(spec.Z)
    dm.set_lattice_spacing(spec.spacing)
    dm.set_particles_per_site(pps)
    dm.set_bytes_per_particle(spec.bytes_per_slot)
    DF = np.asarray(spec.DF).reshape(spec.nst, spec.nst, spec.ns)
    for via in range(spec.nst):
        for to in range(spec.nst):
            for p in range(spec.ns):
                dm.add_diffusion_matrix(float(DF[via, to, p]))
    RL = np.asarray(spec.RL).reshape(spec.nr, spec.nst)
    for r in range(spec.nr):
        for s in range(spec.nst):
            dm.add_reaction_location_matrix(int(RL[r, s]))
    cls = lm.ByteLattice if spec.bytes_per_slot == 1 else lm.IntLattice
    lattice = cls(spec.X, spec.Y, spec.Z, spec.spacing, pps)
    slots = configs.native_to_slots(spec.lattice, spec.X, spec.Y, spec.Z, spec.slots, spec.bytes_per_slot)
    sites = spec.sites.reshape(spec.Z, spec.Y, spec.X)
    lattice.getSiteLatticeView()[:] = sites
    for i in np.nonzero(slots.any(axis=1))[0]:
        x, y, z = i % spec.X, (i // spec.X) % spec.Y, i // (spec.X * spec.Y)
        for p in slots[i]:
            if p:
                lattice.addParticle(int(x), int(y), int(z), int(p))
    return rm, dm, lattice, init


def write_jlm_file(lm, path, spec, pps, params):
    """LmWriteMixin.finalize's lm calls: create, open, models, lattice,
    parameters, close."""
    rm, dm, lattice, init = _jlm_model(lm, spec, pps)
    lm.SimulationFile.create(path)
    f = lm.SimulationFile(path)
    f.setReactionModel(rm)
    f.setDiffusionModel(dm)
    f.setSpatialModel(lm.SpatialModel())
    f.setDiffusionModelLattice(dm, lattice)
    for k, v in params.items():
        f.setParameter(k, v)
    f.close()
    return lattice, init


def test_import_lm_and_jlm_file(tmp_path):
    import lattice_microbes_b200.lm as mod
    import lm
    assert lm is mod
    assert lm.getCompiledLatticeMaxOccupancy() == 16
    spec = configs.config0(seed=3, edge=16, nA=300, nB=200)
    path = str(tmp_path / "jlm.lm")
    params = {"writeInterval": "20", "latticeWriteInterval": "40", "maxTime": "5.0000000000e-03",
              "timestep": "5.0000000000e-05", "hookInterval": ""}
    lattice, init = write_jlm_file(lm, path, spec, 16, params)
    from lattice_microbes_b200.lmfile import LMFile
    with LMFile(path) as f:
        for k, v in params.items():
            assert f.getParameter(k) == v
        r = f.reaction_model()
        assert r["numberSpecies"] == spec.ns and r["numberReactions"] == spec.nr
        assert list(r["initialSpeciesCounts"]) == list(init)
        assert [x["type"] for x in r["reactions"]] == list(spec.rtype)
        assert np.array_equal(np.asarray(r["stoichiometricMatrix"]).reshape(spec.ns, spec.nr),
                              np.asarray(spec.S).reshape(spec.ns, spec.nr))
        d = f.diffusion_model()
        assert int(d["particlesPerSite"]) == 16
        assert np.allclose(d["DiffusionMatrix"].reshape(-1), np.asarray(spec.DF).reshape(-1))
        p, s = lattice.rowMajor()
        assert np.array_equal(d["Lattice"].reshape(p.shape), p)
        assert np.array_equal(d["LatticeSites"].reshape(s.shape), s)
    f = lm.simulationFile(path)
    f.setParameter("seed", "4242")
    f.close()
    with LMFile(path) as g:
        assert g.getParameter("seed") == "4242"
        assert g.getParameter("timestep") == params["timestep"]
        assert np.array_equal(g.diffusion_model()["Lattice"].reshape(p.shape), p)
    assert lm.SimulationFile.isValidFile(path)
    assert not lm.SimulationFile.isValidFile(str(tmp_path / "absent.lm"))
