"""lm::rdme::MpdRdmeSolver / IntMpdRdmeSolver for Python callers.

pyLM's RDMESimulation and jLM's runSolver drive the reference's SWIG class
(src/swig/lm.i:949-1015) with initialize / buildModel / buildDiffusionModel /
generateTrajectory and subclass it to override hookSimulation and the other
callbacks.  This module gives the same calls, argument meaning and callback
contract on top of the C ABI, so such a script switches by changing the class
it instantiates:

    class Solver(MpdRdmeSolver):
        def hookSimulation(self, time, lattice):
            ...                      # lattice: HostLattice, reference accessors
            return 0                 # 0 / 1 / 2 / 3 as in MpdRdmeSolver

    s = Solver()
    s.initialize(replicate, {"seed": "1234", "timestep": "5e-05", "maxTime": "1.0",
                             "writeInterval": "1000", "latticeWriteInterval": "10000"})
    s.buildModel(ns, nr, init, types, K, S, D)
    s.buildDiffusionModel(nst, DF, RL, X, Y, Z, 8, 1, spacing, lattice_xyzp, sites_xyz)
    s.generateTrajectory()

Outputs go to writeSpeciesCounts / writeLattice / writeLatticeSites, which by
default keep the records in memory (speciesCounts, latticeFrames); the
reference sends the same records to its HDF5 output queue.
"""
import time as _time

import numpy as np

from . import _lib as L
from .solver import Context, Lattice, Model, compose_seed


def trajectory_events(total, counts_interval, lattice_interval, hook_interval=None):
    """The timesteps after which MpdRdmeSolver::generateTrajectory
    (MpdRdmeSolver.cu:485-668) does something, with what it does there:
    yields (step, hook, lattice, counts) for each such step, in order, for a
    run of `total` timesteps.  Intervals are in timesteps; an interval of 0
    fires after every timestep, as in the reference; hook_interval None means
    no hook."""
    next_counts, next_lattice = counts_interval, lattice_interval
    next_hook = hook_interval if hook_interval is not None else None
    step = 0
    while step < total:
        ev = total
        ev = min(ev, next_counts if next_counts > step else step + 1)
        ev = min(ev, next_lattice if next_lattice > step else step + 1)
        if next_hook is not None:
            ev = min(ev, next_hook if next_hook > step else step + 1)
        step = ev
        hook = next_hook is not None and step >= next_hook
        lat = step >= next_lattice
        cnt = step >= next_counts
        if hook:
            next_hook += hook_interval
        if lat:
            next_lattice += lattice_interval
        if cnt:
            next_counts += counts_interval
        if hook or lat or cnt:
            yield step, hook, lat, cnt


def timesteps_for(max_time, tau):
    """Timesteps the reference runs: it loops while timestep * tau < maxTime."""
    if tau <= 0.0:
        return 0
    n = int(np.floor(max_time / tau))
    while n * tau < max_time:
        n += 1
    while n > 0 and (n - 1) * tau >= max_time:
        n -= 1
    return n


class HostLattice:
    """Host copy of a lattice in the native layout, with the reference
    lattice's accessors (rdme/Lattice.h:131-259, ByteLattice / IntLattice
    views of lm.i:854-915).  `particles` is the native word-planar array
    (word w of site i = x + y X + z X Y at particles[w N + i]; a ByteLattice
    word holds 4 slots), `sites` the [z][y][x] site types."""

    def __init__(self, X, Y, Z, slots, bytes_per_particle, spacing=0.0):
        self.X, self.Y, self.Z, self.slots = X, Y, Z, slots
        self.bytes_per_particle = bytes_per_particle
        self.spacing = spacing
        self.words = slots // 4 if bytes_per_particle == 1 else slots
        self.particles = np.zeros(self.words * X * Y * Z, dtype=np.uint32)
        self.sites = np.zeros(X * Y * Z, dtype=np.uint8)

    # Lattice (rdme/Lattice.h)
    def getXSize(self):
        return self.X

    def getYSize(self):
        return self.Y

    def getZSize(self):
        return self.Z

    def getSize(self):
        return (self.X, self.Y, self.Z)

    def getNumberSites(self):
        return self.X * self.Y * self.Z

    def getSpacing(self):
        return self.spacing

    def getMaxOccupancy(self):
        return self.slots

    def _index(self, x, y, z):
        if not (0 <= x < self.X and 0 <= y < self.Y and 0 <= z < self.Z):
            raise IndexError("site (%d, %d, %d) outside the lattice" % (x, y, z))
        return x + y * self.X + z * self.X * self.Y

    def getSiteType(self, x, y, z):
        return int(self.sites[self._index(x, y, z)])

    def setSiteType(self, x, y, z, site_type):
        self.sites[self._index(x, y, z)] = site_type

    def getParticle(self, x, y, z, index):
        if not 0 <= index < self.slots:
            raise IndexError("particle index %d" % index)
        i, N = self._index(x, y, z), self.getNumberSites()
        if self.bytes_per_particle == 1:
            return int((self.particles[(index // 4) * N + i] >> np.uint32(8 * (index % 4))) & np.uint32(0xFF))
        return int(self.particles[index * N + i])

    def getOccupancy(self, x, y, z):
        n = 0
        while n < self.slots and self.getParticle(x, y, z, n) != 0:
            n += 1
        return n

    def _set_slot(self, i, index, value):
        N = self.getNumberSites()
        if self.bytes_per_particle == 1:
            k, sh = (index // 4) * N + i, np.uint32(8 * (index % 4))
            w = self.particles[k] & ~(np.uint32(0xFF) << sh)
            self.particles[k] = w | (np.uint32(value & 0xFF) << sh)
        else:
            self.particles[index * N + i] = value

    def addParticle(self, x, y, z, particle):
        """ByteLattice::addParticle: the first free slot; raises when full
        (InvalidParticleException in the reference)."""
        n = self.getOccupancy(x, y, z)
        if n >= self.slots:
            raise ValueError("site (%d, %d, %d) is full" % (x, y, z))
        self._set_slot(self._index(x, y, z), n, particle)

    def removeParticles(self, x, y, z):
        i = self._index(x, y, z)
        for k in range(self.slots):
            self._set_slot(i, k, 0)

    def getParticleCounts(self):
        """{species: count} over the lattice (ByteLattice.cpp:495-520)."""
        if self.bytes_per_particle == 1:
            v = self.particles.view(np.uint8)
        else:
            v = self.particles
        ids, counts = np.unique(v[v != 0], return_counts=True)
        return {int(s): int(c) for s, c in zip(ids, counts)}

    def rowMajor(self):
        """(particles [x][y][z][p], site types [x][y][z]): the arrays
        buildDiffusionModel takes, as Lattice::rowMajorByteSerialize /
        rowMajorIntSerialize and rowMajorByteSerializeSites lay them out."""
        v = self.getParticleLatticeView()                    # (words, Z, Y, X, per-word slots)
        p = np.moveaxis(v, 0, 3).reshape(self.Z, self.Y, self.X, self.slots)
        return (np.ascontiguousarray(p.transpose(2, 1, 0, 3)),
                np.ascontiguousarray(self.getSiteLatticeView().transpose(2, 1, 0)))

    # Views (lm.i:894-895, 913-914)
    def getSiteLatticeView(self):
        """Site types, shape (Z, Y, X), sharing memory with the lattice."""
        return self.sites.reshape(self.Z, self.Y, self.X)

    def getParticleLatticeView(self):
        """Particles, shape (words, Z, Y, X, per-word slots): uint8 with 4
        slots per word for ByteLattices, uint32 with 1 for IntLattices;
        shares memory with the lattice."""
        if self.bytes_per_particle == 1:
            return self.particles.view(np.uint8).reshape(self.words, self.Z, self.Y, self.X, 4)
        return self.particles.reshape(self.words, self.Z, self.Y, self.X, 1)


def getCompiledLatticeMaxOccupancy():
    """lm.getCompiledLatticeMaxOccupancy (lm.i:854): the particles per site
    pyLM and jLM give new lattices -- 16, the reference build's default
    MPD_LATTICE_MAX_OCCUPANCY (src/cmake/options.cmake:61).  The solvers here
    take 4, 8, 16 or 32 slots per site on a ByteLattice and 4, 8 or 16 on an
    IntLattice, chosen per lattice at run time."""
    return 16


class ByteLattice(HostLattice):
    """lm.ByteLattice(xSize, ySize, zSize, spacing, particlesPerSite)."""

    def __init__(self, xSize, ySize, zSize, spacing, particlesPerSite):
        super().__init__(xSize, ySize, zSize, particlesPerSite, 1, spacing)


class IntLattice(HostLattice):
    """lm.IntLattice(xSize, ySize, zSize, spacing, particlesPerSite)."""

    def __init__(self, xSize, ySize, zSize, spacing, particlesPerSite):
        super().__init__(xSize, ySize, zSize, particlesPerSite, 4, spacing)


class MpdRdmeSolver:
    """lm::rdme::MpdRdmeSolver (ByteLattice); IntMpdRdmeSolver below."""

    bytes_per_particle = 1
    tracks_max_counts = True

    def __init__(self, device=0):
        self.ctx = Context(device)
        self.model = None
        self.lat = None
        self.parameters = {}
        self.replicate = 0
        self.seed = 0
        self.overflow_mode = L.LMB_OVERFLOW_CLASSIC
        self.lattice = None
        self.speciesCounts = []       # (time, counts of species 1..ns)
        self.latticeFrames = []       # (time, particles copy, sites copy)
        self.maxParticleCounts = None  # per species id (index 0 unused)
        self.maxSiteCounts = None      # per site type (type 0 not counted)
        self.lastRunStats = None
        self._run_counts = None       # species totals the last run took (None: take them anew)
        self.output = None            # lmfile.LMFileWriter the trajectory goes to
        self._write_inputs = False
        self.checkpointInterval = 0.0  # seconds between checkpoints of the output file (0: none)
        self._last_checkpoint = 0.0
        self._stop = False

    def needsReactionModel(self):
        return True

    def needsDiffusionModel(self):
        return True

    # ---- set-up (MpdRdmeSolver.cu:107-162, CMESolver.h:200-201, RDMESolver.cpp:97-189)
    def initialize(self, replicate, parameters):
        """seed = (seedTop << 16) | (replicate & 0xFFFF), seedTop from the
        "seed" parameter (the clock's nanoseconds when 0);
        "rdme.mpd.overflowhandler" classic (default) or relaxed."""
        self.replicate = replicate
        self.parameters = {k: str(v) for k, v in dict(parameters).items()}
        seed_top = int(float(self.parameters.get("seed", "0") or 0))
        if seed_top == 0:
            seed_top = _time.time_ns() % 1000000000
        self.seed = compose_seed(seed_top, replicate)
        handler = self.parameters.get("rdme.mpd.overflowhandler", "classic")
        self.overflow_mode = L.LMB_OVERFLOW_RELAXED if handler == "relaxed" else L.LMB_OVERFLOW_CLASSIC

    def buildModel(self, numberSpecies, numberReactions, initialSpeciesCounts, reactionTypes, K, S, D, kCols=1):
        """Reaction types 0..3; K [R * kCols] (column 0 used); S and D
        species-major [NS * R]."""
        self._ns, self._nr = int(numberSpecies), int(numberReactions)
        K = np.asarray(K, dtype=np.float64).reshape(-1)
        self._rtype = np.asarray(reactionTypes, dtype=np.uint32).reshape(-1)
        self._K = K[::int(kCols)][:self._nr] if self._nr else np.zeros(0)
        self._K_rows = K.reshape(-1, int(kCols))[:self._nr] if self._nr else np.zeros((0, 1))
        self._S = np.asarray(S, dtype=np.int32).reshape(-1)
        self._D = np.asarray(D, dtype=np.uint32).reshape(-1)
        self._initial = np.asarray(initialSpeciesCounts, dtype=np.uint32).reshape(-1)

    def buildDiffusionModel(self, numberSiteTypes, DF, RL, X, Y, Z, particlesPerSite, bytesPerParticle,
                            latticeSpacing, latticeData, latticeSitesData, rowMajorData=True):
        """DF [NST * NST * NS] m^2/s, RL [R * NST]; lattice [x][y][z][p] and
        site types [x][y][z] row-major; "timestep" from the parameters."""
        if not rowMajorData:
            raise ValueError("columns major lattice data is not currently supported")
        if bytesPerParticle != self.bytes_per_particle:
            raise ValueError("bytes_per_particle does not match the solver's lattice type")
        self._nst = int(numberSiteTypes)
        self.tau = float(self.parameters.get("timestep", "0"))
        spec = _ModelInputs(self._ns, self._nst, self._nr, self._rtype, self._K, self._S, self._D,
                            np.asarray(DF, dtype=np.float64).reshape(-1),
                            np.asarray(RL, dtype=np.uint32).reshape(-1), self.tau, float(latticeSpacing), X, Y, Z)
        for h in (self.lat, self.model):
            if h is not None:
                h.close()
        self.model = Model.from_spec(self.ctx, spec)
        self.lat = Lattice(self.ctx, X, Y, Z, particlesPerSite, bytesPerParticle)
        self.lat.set_row_major(latticeData, latticeSitesData, self._ns, self._nst)
        self.lattice = HostLattice(X, Y, Z, particlesPerSite, bytesPerParticle, float(latticeSpacing))
        self._DF = spec.DF
        self._RL = spec.RL

    def setReactionRate(self, rxid, rate):
        """MpdRdmeSolver::setReactionRate: used from the next timestep on."""
        self.model.set_reaction_rate(rxid, rate)

    def setOutputFile(self, writer, writeInputs=True):
        """Writes the trajectory into a `.lm` file (an lmfile.LMFileWriter),
        as the reference's output queue writes it into the simulation file
        (core/LocalDataOutputWorker.cpp): this replicate's species counts,
        lattice frames (from the device, through the writer's thread), site
        frames and, for the byte lattice, the max counts.  With writeInputs
        the parameters, both models and the initial lattice go in too when
        the trajectory starts (what pyLM writes before it runs a solver).
        The caller closes the writer."""
        self.output = writer
        self._write_inputs = bool(writeInputs)

    def _maybe_checkpoint(self):
        # CheckpointSignaler (core/CheckpointSignaler.cpp:72-180): every
        # checkpointInterval seconds of wall time the file is checkpointed
        # (here at the next record written).
        if self.output is None or self.checkpointInterval <= 0:
            return
        now = _time.monotonic()
        if now - self._last_checkpoint >= self.checkpointInterval:
            self.output.checkpoint()
            self._last_checkpoint = now

    def _write_inputs_to_file(self):
        w = self.output
        for k, v in self.parameters.items():
            w.set_parameter(k, v)
        w.set_reaction_model(self._initial, self._rtype, [list(r) for r in self._K_rows],
                             self._S.reshape(self._ns, self._nr), self._D.reshape(self._ns, self._nr))
        DF = self._DF.reshape(self._nst, self._nst, self._ns)
        w.set_diffusion_model(self.lattice.spacing, self.lattice.X, self.lattice.Y, self.lattice.Z, self.lattice.slots,
                              self.bytes_per_particle, DF, self._RL.reshape(self._nr, self._nst))
        p, s = self.lat.get_row_major()
        w.set_diffusion_model_lattice(p, s)

    def _write_sites_to_file(self, time):
        L = self.lattice
        self.output.append_sites(self.replicate, time, L.sites.reshape(L.Z, L.Y, L.X).transpose(2, 1, 0))

    # ---- callbacks (MpdRdmeSolver.cu:789-822); override in a subclass
    def hookSimulation(self, time, lattice):
        return 0

    def onBeginTrajectory(self, lattice):
        return 0

    def onEndTrajectory(self, lattice):
        return 0

    def onWriteLattice(self, time, lattice):
        return 0

    # ---- outputs (the reference's output-queue data sets)
    def writeSpeciesCounts(self, time, counts):
        self.speciesCounts.append((time, counts))

    def writeLattice(self, time, lattice):
        self.latticeFrames.append((time, lattice.particles.copy(), lattice.sites.copy()))

    def writeLatticeSites(self, time, lattice):
        pass

    def writeMaxCounts(self, maxParticleCounts, maxSiteCounts):
        """MpdRdmeSolver::writeMaxCounts (MpdRdmeSolver.cu:921-932), at the
        end of the trajectory: per species id the largest count seen at the
        start and at each lattice write; per site type the largest number of
        sites seen at the start and at each site write."""
        self.maxParticleCounts = maxParticleCounts
        self.maxSiteCounts = maxSiteCounts

    # ---- the trajectory
    def _download(self):
        p, s = self.lat.get_native()
        self.lattice.particles[:] = p
        self.lattice.sites[:] = s

    def _upload(self, with_sites):
        self.lat.set_native(self.lattice.particles, self.lattice.sites if with_sites else None)
        self._run_counts = None

    def _species_counts(self):
        """The lattice's species totals: those the last run took, unless the
        lattice was changed since."""
        if self._run_counts is not None:
            return self._run_counts.copy()
        return self.lat.species_counts(self._ns)

    def _record_counts(self, time):
        c = self._species_counts()
        self.writeSpeciesCounts(time, np.asarray(c[1:], dtype=np.uint64))
        if self.output is not None:
            self.output.append_species_counts(self.replicate, [time],
                                              np.asarray(c[1:], dtype=np.int64).astype(np.int32)[None, :])
            self._maybe_checkpoint()

    def _write_lattice(self, time):
        # writeLatticeData (MpdRdmeSolver.cu:854-883): the particle maxima,
        # then the frame.
        c = np.asarray(self._species_counts(), dtype=np.uint32)
        c[0] = 0
        np.maximum(self._max_particles, c, out=self._max_particles)
        if self.output is not None:
            self.output.append_lattice_device(self.replicate, time, self.lat)
        self.writeLattice(time, self.lattice)

    def _update_site_maxima(self):
        t = self.lattice.sites
        c = np.bincount(t[(t > 0) & (t < self._nst)], minlength=self._nst)[:self._nst].astype(np.uint32)
        np.maximum(self._max_sites, c, out=self._max_sites)

    def _hook(self, time):
        r = self.hookSimulation(time, self.lattice)
        if r == 0:
            return
        if r == 1:
            self._upload(False)
        elif r == 2:
            self._upload(True)
            self._update_site_maxima()
            if self.output is not None:
                self._write_sites_to_file(time)
            self.writeLatticeSites(time, self.lattice)
        elif r == 3:
            self._update_site_maxima()
            if self.output is not None:
                self._write_sites_to_file(time)
            self.writeLatticeSites(time, self.lattice)
            self._stop = True
        else:
            raise RuntimeError("Unknown hook return value")

    def generateTrajectory(self):
        """MpdRdmeSolver::generateTrajectory (MpdRdmeSolver.cu:485-668): runs
        timesteps while timestep * tau < maxTime; after a timestep that
        reaches the next hook, lattice-write or species-write step, calls the
        hook, writes the lattice, records the counts, in that order.  Counts
        and lattice are also written at t = 0.  Timesteps between two such
        steps run as one call."""
        p = self.parameters
        counts_interval = int(float(p.get("writeInterval", "0") or 0))
        lattice_interval = int(float(p.get("latticeWriteInterval", "0") or 0))
        hook_interval = int(float(p["hookInterval"])) if p.get("hookInterval", "") != "" else None
        max_time = float(p.get("maxTime", "0") or 0)
        self._stop = False
        self._run_counts = None
        self._download()
        self.onBeginTrajectory(self.lattice)
        self._upload(True)
        if self.output is not None and self._write_inputs:
            self._write_inputs_to_file()
        self._last_checkpoint = _time.monotonic()
        t = 0.0
        self._max_particles = np.zeros(self._ns + 1, dtype=np.uint32)
        self._max_sites = np.zeros(self._nst, dtype=np.uint32)
        self._record_counts(t)
        self._write_lattice(t)
        self._update_site_maxima()  # initMaxCounts (MpdRdmeSolver.cu:548, 824-850)
        self._hook(t)
        total = timesteps_for(max_time, self.tau)
        done = 0
        for step, hook, lat, cnt in trajectory_events(total, counts_interval, lattice_interval, hook_interval):
            if self._stop:
                break
            if (cnt or lat) and not hook:
                # The totals a record needs, taken in the run's own work.
                _, self.lastRunStats, self._run_counts = self.lat.run_counts(
                    self.model, self.seed, done, step - done, self._ns, self.overflow_mode)
            else:
                _, self.lastRunStats = self.lat.run(self.model, self.seed, done, step - done, self.overflow_mode)
                self._run_counts = None
            done = step
            t = step * self.tau
            if hook:
                self._download()
                self._hook(t)
            if lat:
                self._download()
                if self.onWriteLattice(t, self.lattice):
                    self._upload(True)
                self._write_lattice(t)
            if cnt:
                self._record_counts(t)
        if not self._stop and done < total:
            _, self.lastRunStats = self.lat.run(self.model, self.seed, done, total - done, self.overflow_mode)
        self._download()
        self.onEndTrajectory(self.lattice)
        if self.tracks_max_counts:
            if self.output is not None:
                self.output.write_max_counts(self.replicate, self._max_particles, self._max_sites)
            self.writeMaxCounts(self._max_particles.copy(), self._max_sites.copy())

    def close(self):
        for h in (self.lat, self.model):
            if h is not None:
                h.close()
        self.lat = self.model = None
        self.ctx.close()


class IntMpdRdmeSolver(MpdRdmeSolver):
    """lm::rdme::IntMpdRdmeSolver: the same solver on an IntLattice."""

    bytes_per_particle = 4
    # IntMpdRdmeSolver::generateTrajectory keeps no maxima (its initMaxCounts
    # call is disabled, IntMpdRdmeSolver.cu:617) and writes none.
    tracks_max_counts = False


def runSolver(simulationFilename, replicate, solver, cudaDevices=None, checkpointInterval=0):
    """lm.runSolver (core/runSimulation.cpp:130-260), as pyLM's
    RDMESimulation.runSolver and jLM call it per replicate: reads the
    parameters, the reaction model and the diffusion model with its lattice
    from the `.lm` file, initializes `solver` (an MpdRdmeSolver or
    IntMpdRdmeSolver, or a subclass) for `replicate`, runs
    generateTrajectory and writes the replicate's records into the same
    file.  The file's existing contents, earlier replicates included, are
    carried over: the new file is written beside it and replaces it when the
    run ends.  Like the reference, an exception raised by the run is printed
    and the records written so far are kept.  With `checkpointInterval` > 0
    the file so far is copied, complete, to "<file>.chk" every that many
    seconds (at the next record), as the reference's CheckpointSignaler has
    it done; the copy is of the file being written beside the original.
    `cudaDevices` is accepted for the reference's signature; the solver runs
    on its own device."""
    import os
    import sys

    from .lmfile import LMFile, LMFileWriter
    with LMFile(simulationFilename) as f:
        params = f.parameters()
        rm = f.reaction_model() if solver.needsReactionModel() else None
        dm = f.diffusion_model() if solver.needsDiffusionModel() else None
    solver.initialize(replicate, params)
    if rm is not None:
        ns, nr = rm["numberSpecies"], rm["numberReactions"]
        K = np.full((nr, 10), np.nan)
        for i, r in enumerate(rm["reactions"]):
            K[i, :len(r["rateConstants"])] = r["rateConstants"]
        init = rm["initialSpeciesCounts"] or [0] * ns
        solver.buildModel(ns, nr, init, [r["type"] for r in rm["reactions"]], K.ravel(),
                          rm["stoichiometricMatrix"], rm["dependencyMatrix"], kCols=10)
    if dm is not None:
        nst = int(dm["numberSiteTypes"])
        bpp = int(dm.get("bytes_per_particle", 1))
        RL = dm.get("ReactionLocationMatrix", np.zeros((0, nst), np.uint32))
        solver.buildDiffusionModel(nst, dm["DiffusionMatrix"].ravel(), np.asarray(RL).ravel(),
                                   int(dm["latticeXSize"]), int(dm["latticeYSize"]), int(dm["latticeZSize"]),
                                   int(dm["particlesPerSite"]), bpp, float(dm["latticeSpacing"]),
                                   dm["Lattice"].reshape(-1), dm["LatticeSites"].reshape(-1))
    tmp = "%s.%d.tmp" % (simulationFilename, os.getpid())
    w = LMFileWriter(tmp)
    w.checkpoint_path = simulationFilename + ".chk"
    try:
        with LMFile(simulationFilename) as f:
            w.copy_from(f)
        solver.setOutputFile(w, writeInputs=False)
        solver.checkpointInterval = float(checkpointInterval or 0)
        try:
            solver.generateTrajectory()
        except Exception as e:  # runSimulation.cpp:228-240: reported, the file is still closed
            print("Exception during execution of replicate: %s." % e, file=sys.stderr)
        solver.output = None
        w.close()
    except BaseException:
        if w.h:
            w.close()
        os.unlink(tmp)
        raise
    os.replace(tmp, simulationFilename)


class _ModelInputs:
    """The fields Model.from_spec reads."""

    def __init__(self, ns, nst, nr, rtype, K, S, D, DF, RL, tau, spacing, X, Y, Z):
        self.ns, self.nst, self.nr = ns, nst, nr
        self.rtype, self.K, self.S, self.D, self.DF, self.RL = rtype, K, S, D, DF, RL
        self.tau, self.spacing = tau, spacing
        self.X, self.Y, self.Z = X, Y, Z
