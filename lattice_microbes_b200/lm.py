"""The `lm` module of pyLM and jLM scripts, on this package.

jLM and pyLM import `lm` (the reference's SWIG module, src/swig/lm.i) for
the lattice classes, the solver classes, the protobuf model messages they
fill, SimulationFile and runSolver.  Importing this module makes it that
`lm` for the process, unless a module of that name is already loaded:

    import lattice_microbes_b200.lm   # once, before the script's `import lm`
    import lm

What it carries, each with the reference's names, arguments and meaning:

* MpdRdmeSolver, IntMpdRdmeSolver, ByteLattice, IntLattice,
  getCompiledLatticeMaxOccupancy, runSolver (lm.i:854-1042);
* ReactionModel, DiffusionModel, SpatialModel: the message calls jLM's
  LmWriteMixin makes to build a model (jlm/jLM/LmInteract.py:230-335);
* SimulationFile (lm.i:716-746): create, isValidFile, and an open file whose
  setParameter / setReactionModel / setDiffusionModel /
  setDiffusionModelLattice / setSpatialModel / getters and close are those of
  io/hdf5/SimulationFile.  jLM's Sim.run calls `lm.simulationFile(name)`
  (jlm/jLM/RDME.py:451), a name lm.i does not define; here it is
  SimulationFile.

An open SimulationFile writes beside the file and replaces it at close, as
runSolver does: the existing contents are carried over and what was set
replaces what was there.
"""
import os
import sys

import numpy as np

from .lmfile import LMFile, LMFileWriter
from .rdme import (ByteLattice, IntLattice, IntMpdRdmeSolver, MpdRdmeSolver, getCompiledLatticeMaxOccupancy,
                   runSolver)

__all__ = ["MpdRdmeSolver", "IntMpdRdmeSolver", "ByteLattice", "IntLattice", "getCompiledLatticeMaxOccupancy",
           "runSolver", "ReactionModel", "DiffusionModel", "SpatialModel", "SimulationFile", "simulationFile",
           "BUILD_CONFIGURATION"]

BUILD_CONFIGURATION = ("lattice_microbes_b200: MPD-RDME on sm_100a (B200); ByteLattice 4/8/16/32 and IntLattice "
                       "4/8/16 particles per site chosen per lattice; compiled lattice max occupancy %d"
                       % getCompiledLatticeMaxOccupancy())


class _Reaction:
    """ReactionModel_Reaction (lm.i:680-690): a reaction's type and rate
    constants."""

    def __init__(self):
        self._type = 0
        self._k = []

    def set_type(self, t):
        self._type = int(t)

    def type(self):
        return self._type

    def add_rate_constant(self, k):
        self._k.append(float(k))

    def rate_constant(self, i):
        return self._k[i]

    def rate_constant_size(self):
        return len(self._k)


class ReactionModel:
    """lm::io::ReactionModel (protobuf/ReactionModel.proto), the calls jLM and
    pyLM make: counts, reactions, and the species-major stoichiometry and
    dependency matrices ([species][reaction], one entry per add call)."""

    def __init__(self):
        self._nr = 0
        self._ns = 0
        self._init = []
        self._rx = []
        self._S = []
        self._D = []

    def set_number_reactions(self, n):
        self._nr = int(n)

    def number_reactions(self):
        return self._nr

    def set_number_species(self, n):
        self._ns = int(n)

    def number_species(self):
        return self._ns

    def add_initial_species_count(self, c):
        self._init.append(int(c))

    def add_reaction(self):
        self._rx.append(_Reaction())

    def reaction(self, r):
        return self._rx[r]

    def mutable_reaction(self, r):
        return self._rx[r]

    def add_stoichiometric_matrix(self, v):
        self._S.append(int(v))

    def add_dependency_matrix(self, v):
        self._D.append(int(v))

    def _arrays(self):
        ns, nr = self._ns, self._nr
        if len(self._rx) != nr or len(self._S) != ns * nr or len(self._D) != ns * nr:
            raise ValueError("reaction model incomplete: %d reactions, %d stoichiometric and %d dependency "
                             "entries for %d species x %d reactions" % (len(self._rx), len(self._S), len(self._D),
                                                                        ns, nr))
        init = self._init if self._init else [0] * ns
        return (np.asarray(init, np.uint32), np.asarray([r.type() for r in self._rx], np.uint32),
                [list(r._k) for r in self._rx], np.asarray(self._S, np.int32).reshape(ns, nr),
                np.asarray(self._D, np.uint32).reshape(ns, nr))


class DiffusionModel:
    """lm::io::DiffusionModel (protobuf/DiffusionModel.proto), the calls jLM
    makes: sizes, spacing, occupancy, the diffusion matrix [via][to][species]
    and the reaction location matrix [reaction][site type], one entry per add
    call."""

    def __init__(self):
        self._f = dict(number_reactions=0, number_species=0, number_site_types=0, lattice_x_size=0,
                       lattice_y_size=0, lattice_z_size=0, lattice_spacing=0.0, particles_per_site=0,
                       bytes_per_particle=1)
        self._DF = []
        self._RL = []

    def __getattr__(self, name):
        f = self.__dict__.get("_f")
        if f is not None:
            if name.startswith("set_") and name[4:] in f:
                return lambda v, k=name[4:]: f.__setitem__(k, type(f[k])(v))
            if name in f:
                return lambda k=name: f[k]
        raise AttributeError(name)

    def add_diffusion_matrix(self, v):
        self._DF.append(float(v))

    def add_reaction_location_matrix(self, v):
        self._RL.append(int(v))

    def _arrays(self):
        f = self._f
        nst, ns, nr = f["number_site_types"], f["number_species"], f["number_reactions"]
        if len(self._DF) != nst * nst * ns or len(self._RL) != nr * nst:
            raise ValueError("diffusion model incomplete: %d diffusion and %d location entries for %d site types, "
                             "%d species, %d reactions" % (len(self._DF), len(self._RL), nst, ns, nr))
        return (np.asarray(self._DF, np.float64).reshape(nst, nst, ns),
                np.asarray(self._RL, np.uint32).reshape(nr, nst))


class SpatialModel:
    """lm::io::SpatialModel; jLM hands over an empty one."""


class SimulationFile:
    """lm::io::hdf5::SimulationFile (lm.i:716-746) on a `.lm` file."""

    @staticmethod
    def create(filename):
        """SimulationFile::create: a new, empty `.lm` file; refuses an
        existing one."""
        LMFileWriter(filename).close()

    @staticmethod
    def isValidFile(filename):
        try:
            with LMFile(filename):
                return True
        except Exception:
            return False

    def __init__(self, filename):
        self.filename = os.fspath(filename)
        self._tmp = "%s.%d.%d.tmp" % (self.filename, os.getpid(), id(self))
        with LMFile(self.filename) as f:
            self._writer = LMFileWriter(self._tmp)
            try:
                self._writer.copy_from(f)
            except BaseException:
                self._writer.close()
                os.unlink(self._tmp)
                raise
        self._params = {}

    def _w(self):
        if self._writer is None:
            raise ValueError("SimulationFile %s is closed" % self.filename)
        return self._writer

    def setParameter(self, key, value):
        self._w().set_parameter(str(key), str(value))
        self._params[str(key)] = str(value)

    def getParameter(self, key, default=""):
        if key in self._params:
            return self._params[key]
        with LMFile(self.filename) as f:
            return f.getParameter(key, default)

    def setReactionModel(self, rm):
        init, types, k, S, D = rm._arrays()
        self._w().set_reaction_model(init, types, k, S, D)

    def setDiffusionModel(self, dm):
        DF, RL = dm._arrays()
        self._w().set_diffusion_model(dm.lattice_spacing(), dm.lattice_x_size(), dm.lattice_y_size(),
                                      dm.lattice_z_size(), dm.particles_per_site(), dm.bytes_per_particle(), DF,
                                      RL)

    def setDiffusionModelLattice(self, dm, lattice):
        """The lattice (lm.ByteLattice or lm.IntLattice) as the model's
        initial state, row-major as SimulationFile writes it."""
        if (lattice.getXSize(), lattice.getYSize(), lattice.getZSize()) != (
                dm.lattice_x_size(), dm.lattice_y_size(), dm.lattice_z_size()):
            raise ValueError("lattice size differs from the diffusion model's")
        particles, sites = lattice.rowMajor()
        self._w().set_diffusion_model_lattice(particles, sites)

    def setSpatialModel(self, sm):
        """An empty spatial model writes nothing (jLM's case)."""
        self._w()

    def close(self):
        if self._writer is not None:
            w, self._writer = self._writer, None
            w.close()
            os.replace(self._tmp, self.filename)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # Getters read the file as it is on disk (after close, with the changes).
    def _read(self, name, *a):
        with LMFile(self.filename) as f:
            return getattr(f, name)(*a)

    def getParameters(self):
        return self._read("getParameters")

    def getLatticeTimes(self, replicate):
        return self._read("getLatticeTimes", replicate)

    def getLattice(self, replicate, index):
        return self._read("getLattice", replicate, index)

    def getSpeciesCountTimes(self, replicate):
        return self._read("getSpeciesCountTimes", replicate)

    def getSpeciesCounts(self, replicate):
        return self._read("getSpeciesCounts", replicate)


simulationFile = SimulationFile

sys.modules.setdefault("lm", sys.modules[__name__])
