"""Seeded synthetic MPD-RDME problems with the shapes of the benchmark configs.

Each generator returns a ``ModelSpec`` holding the same inputs the reference
solver receives from a ``.lm`` file or from pyLM/jLM: reaction types and rate
constants in Lattice Microbes units (CMESolver::buildModel), the species-major
stoichiometry and dependency matrices, the diffusion matrix DF[src][dst][sp] in
m^2/s, the reaction-location matrix RL[rxn][site type], the timestep and the
lattice spacing (RDMESolver::buildDiffusionModel), plus a native word-planar
particle lattice and the site-type lattice.

Rate constants follow jLM's conversion to LM units (jlm/jLM/Types.py:306-339):
second-order k_LM = k / (N_A * V_site) / N_sites, first-order k_LM = k,
zeroth-order k_LM = k * N_A * V_site * N_sites, so that the solver's
per-site scaling (MpdRdmeSolver.cu:697-727) gives per-site stochastic rates.

Particle placement follows LatticeBuilder::discretizeTo
(builder/LatticeBuilder.cpp:587-608): a uniformly random site of the requested
type is drawn until one with a free slot is found, and the particle goes into
the first free slot.  The random draws use numpy, not the reference RNG.
"""
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

N_AVOGADRO = 6.02214076e23

# Reaction types (CMESolver.h:79-112).
ZEROTH, FIRST, SECOND, SECOND_SELF = 0, 1, 2, 3


@dataclass
class ModelSpec:
    name: str
    X: int
    Y: int
    Z: int
    slots: int
    bytes_per_slot: int
    ns: int
    nst: int
    tau: float
    spacing: float
    rtype: np.ndarray          # [R] uint32
    K: np.ndarray              # [R] float64 (one rate column)
    S: np.ndarray              # [NS, R] int32, species-major like CMESolver
    D: np.ndarray              # [NS, R] uint32 dependency matrix
    DF: np.ndarray             # [NST, NST, NS] float64
    RL: np.ndarray             # [R, NST] uint32
    lattice: np.ndarray        # [W * N] uint32 native word-planar
    sites: np.ndarray          # [N] uint8, index x + y*X + z*X*Y
    steps: int = 100
    species_names: List[str] = field(default_factory=list)

    @property
    def nr(self):
        return int(len(self.rtype))

    @property
    def words(self):
        return self.slots // 4 if self.bytes_per_slot == 1 else self.slots

    @property
    def nsites(self):
        return self.X * self.Y * self.Z

    def reactants(self):
        """0-based (s1, s2) per reaction from the dependency columns, read as
        CMESolver::buildModel does (CMESolver.cpp:340-430)."""
        s1 = np.zeros(self.nr, dtype=np.uint32)
        s2 = np.zeros(self.nr, dtype=np.uint32)
        for r in range(self.nr):
            deps = np.nonzero(self.D[:, r] == 1)[0]
            if self.rtype[r] == ZEROTH:
                assert len(deps) == 0
            elif self.rtype[r] in (FIRST, SECOND_SELF):
                assert len(deps) == 1
                s1[r] = deps[0]
            elif self.rtype[r] == SECOND:
                assert len(deps) == 2
                s1[r], s2[r] = deps[0], deps[1]
        return s1, s2


def _site_volume_litres(spacing):
    return (spacing ** 3) * 1000.0


def lm_rate(k, order, spacing, nsites):
    """Physical rate constant -> LM units (jlm/jLM/Types.py:318-339)."""
    nav = N_AVOGADRO * _site_volume_litres(spacing)
    conc_power = 1 - order
    return k * nav ** conc_power * float(nsites) ** conc_power


def empty_lattice(X, Y, Z, slots, bytes_per_slot):
    words = slots // 4 if bytes_per_slot == 1 else slots
    return np.zeros(words * X * Y * Z, dtype=np.uint32)


def place_particles(lattice, sites, X, Y, Z, slots, bytes_per_slot, species_id, count,
                    site_type, rng, occupancy=None):
    """Adds ``count`` particles of 1-based ``species_id`` at random sites of
    ``site_type``, retrying full sites, each into the first free slot."""
    N = X * Y * Z
    if occupancy is None:
        occupancy = occupancy_of(lattice, N, slots, bytes_per_slot)
    allowed = np.nonzero(sites == site_type)[0]
    if len(allowed) == 0 and count > 0:
        raise ValueError("no sites of type %d" % site_type)
    remaining = count
    while remaining > 0:
        pick = allowed[rng.integers(0, len(allowed), size=remaining)]
        order = np.argsort(pick, kind="stable")
        ps = pick[order]
        first = np.ones(len(ps), dtype=bool)
        first[1:] = ps[1:] != ps[:-1]
        grp_start = np.maximum.accumulate(np.where(first, np.arange(len(ps)), 0))
        rank = np.arange(len(ps)) - grp_start
        slot = occupancy[ps] + rank
        ok = slot < slots
        ps, slot = ps[ok], slot[ok]
        _set_slots(lattice, N, slots, bytes_per_slot, ps, slot, species_id)
        np.add.at(occupancy, ps, 1)
        remaining -= int(ok.sum())
    return occupancy


def occupancy_of(lattice, N, slots, bytes_per_slot):
    occ = np.zeros(N, dtype=np.int64)
    alive = np.ones(N, dtype=bool)
    for k in range(slots):
        v = slot_values(lattice, N, slots, bytes_per_slot, k)
        alive &= v != 0
        occ += alive
    return occ


def slot_values(lattice, N, slots, bytes_per_slot, k):
    if bytes_per_slot == 1:
        w = lattice[(k // 4) * N:(k // 4 + 1) * N]
        return (w >> np.uint32(8 * (k % 4))) & np.uint32(0xFF)
    return lattice[k * N:(k + 1) * N]


def _set_slots(lattice, N, slots, bytes_per_slot, idx, slot, value):
    if bytes_per_slot == 1:
        word = slot // 4
        shift = (8 * (slot % 4)).astype(np.uint32)
        pos = word * N + idx
        # Several slots of one site can share a word: accumulate unbuffered.
        np.bitwise_or.at(lattice, pos, (np.uint32(value) << shift).astype(np.uint32))
    else:
        lattice[slot * N + idx] = np.uint32(value)


def native_to_slots(lattice, X, Y, Z, slots, bytes_per_slot):
    """[N, S] array of slot values from a native lattice."""
    N = X * Y * Z
    return np.stack([slot_values(lattice, N, slots, bytes_per_slot, k) for k in range(slots)], axis=1)


def species_counts(lattice, N, slots, bytes_per_slot, ns):
    counts = np.zeros(ns + 1, dtype=np.int64)
    for k in range(slots):
        v = slot_values(lattice, N, slots, bytes_per_slot, k)
        counts += np.bincount(v.astype(np.int64), minlength=ns + 1)[: ns + 1]
    counts[0] = 0
    return counts


# --------------------------------------------------------------------------
# Config 0: bimolecular A + B <-> C, 32^3, Byte-8
# --------------------------------------------------------------------------

def config0(seed=1, edge=32, nA=None, nB=None, steps=10000):
    """A + B <-> C on an edge^3 cubic lattice (32 nm, D = 1e-12 m^2/s,
    kf = 1.07e6 /M/s, kr = 0.351 /s, tau = 50 us); 1000 A + 1000 B at 32^3,
    scaled by volume for other edges."""
    X = Y = Z = edge
    N = X * Y * Z
    spacing, tau = 32e-9, 50e-6
    if nA is None:
        nA = int(round(1000 * N / 32768))
    if nB is None:
        nB = int(round(1000 * N / 32768))
    ns, nst = 3, 1
    rtype = np.array([SECOND, FIRST], dtype=np.uint32)
    K = np.array([lm_rate(1.07e6, 2, spacing, N), lm_rate(0.351, 1, spacing, N)])
    S = np.array([[-1, 1], [-1, 1], [1, -1]], dtype=np.int32)
    D = np.array([[1, 0], [1, 0], [0, 1]], dtype=np.uint32)
    DF = np.full((nst, nst, ns), 1e-12)
    RL = np.ones((2, nst), dtype=np.uint32)
    lat = empty_lattice(X, Y, Z, 8, 1)
    sites = np.zeros(N, dtype=np.uint8)
    rng = np.random.default_rng(seed)
    occ = place_particles(lat, sites, X, Y, Z, 8, 1, 1, nA, 0, rng)
    place_particles(lat, sites, X, Y, Z, 8, 1, 2, nB, 0, rng, occ)
    return ModelSpec("bimolecular-%d^3" % edge, X, Y, Z, 8, 1, ns, nst, tau, spacing, rtype, K, S, D,
                     DF, RL, lat, sites, steps, ["A", "B", "C"])


# --------------------------------------------------------------------------
# Config 1: rod-shaped cell oscillator, 64x64x128, Byte-8
# --------------------------------------------------------------------------

def rod_cell_sites(X, Y, Z, radius, shell=1.5):
    """Capsule along z: 0 extracellular, 1 cytoplasm, 2 membrane shell."""
    x = np.arange(X) - (X - 1) / 2.0
    y = np.arange(Y) - (Y - 1) / 2.0
    z = np.arange(Z, dtype=np.float64)
    zc0, zc1 = radius + 1.5, Z - radius - 2.5
    zz, yy, xx = np.meshgrid(z, y, x, indexing="ij")
    zcl = np.clip(zz, zc0, zc1)
    d = np.sqrt(xx ** 2 + yy ** 2 + (zz - zcl) ** 2)
    st = np.zeros((Z, Y, X), dtype=np.uint8)
    st[d < radius] = 2
    st[d < radius - shell] = 1
    return st.reshape(-1)


def config1(seed=1, steps=50000, X=64, Y=64, Z=128):
    """MinD/MinE-style oscillator in a rod cell (16 nm, tau = 25 us):
    species D_ATP, D_ADP, E, DE (membrane), Dm (membrane); 8 reactions with
    membrane-only binding; cytoplasm D = 2.5e-12, membrane D = 1e-14 m^2/s;
    4000 D_ATP + 1400 E placed in the cytoplasm."""
    N = X * Y * Z
    spacing, tau = 16e-9, 25e-6
    ns, nst = 5, 3
    D_ATP, D_ADP, E, DE, DM = 0, 1, 2, 3, 4
    CYT, MEM = 1, 2
    # (type, reactants, products, k physical, site types)
    rx = [
        (FIRST, [D_ADP], [D_ATP], 6.0, [CYT, MEM]),
        (FIRST, [D_ATP], [DM], 20.0, [MEM]),
        (SECOND, [D_ATP, DM], [DM, DM], 5.0e7, [MEM]),
        (SECOND, [E, DM], [DE], 8.0e7, [MEM]),
        (FIRST, [DE], [E, D_ADP], 0.7, [MEM]),
        (SECOND, [E, DE], [DE, E], 1.0e6, [MEM]),
        (FIRST, [DM], [D_ADP], 0.05, [MEM]),
        (SECOND, [D_ADP, E], [D_ATP, E], 1.0e5, [CYT]),
    ]
    R = len(rx)
    rtype = np.array([r[0] for r in rx], dtype=np.uint32)
    order = {ZEROTH: 0, FIRST: 1, SECOND: 2, SECOND_SELF: 2}
    K = np.array([lm_rate(r[3], order[r[0]], spacing, N) for r in rx])
    S = np.zeros((ns, R), dtype=np.int32)
    Dm = np.zeros((ns, R), dtype=np.uint32)
    RL = np.zeros((R, nst), dtype=np.uint32)
    for j, (t, re, pr, k, locs) in enumerate(rx):
        for s in re:
            S[s, j] -= 1
            Dm[s, j] = 1
        for s in pr:
            S[s, j] += 1
        for st in locs:
            RL[j, st] = 1
    Dcyt, Dmem = 2.5e-12, 1e-14
    DF = np.zeros((nst, nst, ns))
    for sp in (D_ATP, D_ADP, E):
        for a in (CYT, MEM):
            for b in (CYT, MEM):
                DF[a, b, sp] = Dcyt
    for sp in (DE, DM):
        DF[MEM, MEM, sp] = Dmem
    sites = rod_cell_sites(X, Y, Z, radius=0.45 * min(X, Y))
    lat = empty_lattice(X, Y, Z, 8, 1)
    rng = np.random.default_rng(seed)
    occ = place_particles(lat, sites, X, Y, Z, 8, 1, D_ATP + 1, 4000, CYT, rng)
    place_particles(lat, sites, X, Y, Z, 8, 1, E + 1, 1400, CYT, rng, occ)
    return ModelSpec("rod-cell-%dx%dx%d" % (X, Y, Z), X, Y, Z, 8, 1, ns, nst, tau, spacing, rtype, K,
                     S, Dm, DF, RL, lat, sites, steps, ["D_ATP", "D_ADP", "E", "DE", "Dm"])


# --------------------------------------------------------------------------
# Config 2: crowded large cell, 128x128x256, Int-16
# --------------------------------------------------------------------------

def obstacle_sites(X, Y, Z, fraction, ntypes, rng, rmin=2.0, rmax=6.0):
    """Random spheres of site types 1..ntypes-1 until `fraction` of the
    volume is covered; type 0 is the free cytoplasm (obstacle discretisation
    in the manner of LatticeBuilder.cpp:613-760, not its RNG stream)."""
    st = np.zeros((Z, Y, X), dtype=np.uint8)
    target = fraction * X * Y * Z
    covered = 0
    while covered < target:
        r = rng.uniform(rmin, rmax)
        c = rng.uniform([0, 0, 0], [X, Y, Z])
        t = rng.integers(1, ntypes)
        lo = np.floor(c - r).astype(int)
        hi = np.ceil(c + r).astype(int) + 1
        xs = np.arange(lo[0], hi[0]); ys = np.arange(lo[1], hi[1]); zs = np.arange(lo[2], hi[2])
        zz, yy, xx = np.meshgrid(zs, ys, xs, indexing="ij")
        inside = (xx + 0.5 - c[0]) ** 2 + (yy + 0.5 - c[1]) ** 2 + (zz + 0.5 - c[2]) ** 2 <= r * r
        zi, yi, xi = zz[inside] % Z, yy[inside] % Y, xx[inside] % X
        newly = st[zi, yi, xi] == 0
        covered += int(newly.sum())
        st[zi[newly], yi[newly], xi[newly]] = t
    return st.reshape(-1)


def config2(seed=1, steps=5000, X=128, Y=128, Z=256, ns=200, nr=500, nparticles=1_000_000,
            nst=8, obstacle_fraction=0.20, homodimers=False):
    """200 species, 500 first/second-order reactions with log-uniform rates
    (1e-3..1e2 /s, 1e5..1e7 /M/s), 8 site types (free cytoplasm + 7 obstacle
    classes), per-species D log-uniform in [1e-14, 5e-12] m^2/s (10 nm,
    tau = 10 us), 1M particles in the free cytoplasm, Int lattice, 16 slots.
    Hetero second-order reactions never share a (site type, reactant pair)
    and homodimer reactions are left out unless asked for."""
    rng = np.random.default_rng(seed)
    N = X * Y * Z
    spacing, tau = 10e-9, 10e-6
    sites = obstacle_sites(X, Y, Z, obstacle_fraction, nst, rng)
    Dsp = np.exp(rng.uniform(np.log(1e-14), np.log(5e-12), size=ns))
    DF = np.zeros((nst, nst, ns))
    DF[0, 0, :] = Dsp
    # Species s may also enter and move inside obstacle class 1 + s % 7.
    for s in range(ns):
        t = 1 + s % (nst - 1)
        DF[0, t, s] = DF[t, 0, s] = DF[t, t, s] = Dsp[s] * 0.1
    rtype = np.zeros(nr, dtype=np.uint32)
    K = np.zeros(nr)
    S = np.zeros((ns, nr), dtype=np.int32)
    Dm = np.zeros((ns, nr), dtype=np.uint32)
    RL = np.zeros((nr, nst), dtype=np.uint32)
    pairs = set()
    for j in range(nr):
        second = rng.random() < 0.5
        locs = [0] + [t for t in range(1, nst) if rng.random() < 0.2]
        if second:
            while True:
                a, b = rng.choice(ns, size=2, replace=homodimers)
                key = (min(a, b), max(a, b))
                if a != b and key not in pairs:
                    pairs.add(key)
                    break
                if homodimers and a == b:
                    break
            if a == b:
                rtype[j] = SECOND_SELF
                K[j] = lm_rate(np.exp(rng.uniform(np.log(1e5), np.log(1e7))), 2, spacing, N)
                S[a, j] -= 2
                Dm[a, j] = 1
            else:
                rtype[j] = SECOND
                K[j] = lm_rate(np.exp(rng.uniform(np.log(1e5), np.log(1e7))), 2, spacing, N)
                S[a, j] -= 1
                S[b, j] -= 1
                Dm[a, j] = Dm[b, j] = 1
            S[rng.integers(ns), j] += 1
        else:
            rtype[j] = FIRST
            K[j] = np.exp(rng.uniform(np.log(1e-3), np.log(1e2)))
            a = rng.integers(ns)
            S[a, j] -= 1
            Dm[a, j] = 1
            for p in rng.choice(ns, size=rng.integers(1, 3), replace=False):
                S[p, j] += 1
        for t in locs:
            RL[j, t] = 1
    lat = empty_lattice(X, Y, Z, 16, 4)
    occ = None
    per = np.full(ns, nparticles // ns)
    per[: nparticles - per.sum()] += 1
    for s in range(ns):
        occ = place_particles(lat, sites, X, Y, Z, 16, 4, s + 1, int(per[s]), 0, rng, occ)
    return ModelSpec("crowded-%dx%dx%d" % (X, Y, Z), X, Y, Z, 16, 4, ns, nst, tau, spacing, rtype, K,
                     S, Dm, DF, RL, lat, sites, steps)


# --------------------------------------------------------------------------
# Small randomized problems for parity tests
# --------------------------------------------------------------------------

def random_problem(seed, X=32, Y=16, Z=16, slots=8, bytes_per_slot=1, ns=6, nst=3, nr=8,
                   density=0.5, qmax=0.45, steps=20, zeroth=True, selfrx=True):
    """Dense, multi-type problem exercising every rule: all four reaction
    types, reaction locations, per-type diffusion, full sites (overflows)."""
    rng = np.random.default_rng(seed)
    N = X * Y * Z
    spacing, tau = 1.0, 1.0
    sites = rng.integers(0, nst, size=N).astype(np.uint8)
    DF = rng.uniform(0.0, qmax, size=(nst, nst, ns))
    DF[rng.random(size=DF.shape) < 0.15] = 0.0
    rtype = np.zeros(nr, dtype=np.uint32)
    K = np.zeros(nr)
    S = np.zeros((ns, nr), dtype=np.int32)
    Dm = np.zeros((ns, nr), dtype=np.uint32)
    RL = (rng.random(size=(nr, nst)) < 0.7).astype(np.uint32)
    kinds = [FIRST, SECOND] + ([ZEROTH] if zeroth else []) + ([SECOND_SELF] if selfrx else [])
    pairs = set()
    for j in range(nr):
        t = kinds[j % len(kinds)] if j < len(kinds) else rng.choice(kinds)
        rtype[j] = t
        if t == ZEROTH:
            K[j] = rng.uniform(0.001, 0.02) * N
        elif t == FIRST:
            a = rng.integers(ns)
            S[a, j] -= 1
            Dm[a, j] = 1
            K[j] = rng.uniform(0.01, 0.2)
        elif t == SECOND:
            while True:
                a, b = sorted(rng.choice(ns, size=2, replace=False))
                if (a, b) not in pairs:
                    pairs.add((a, b))
                    break
            S[a, j] -= 1
            S[b, j] -= 1
            Dm[a, j] = Dm[b, j] = 1
            K[j] = rng.uniform(0.01, 0.2) / N
        else:
            a = rng.integers(ns)
            S[a, j] -= 2
            Dm[a, j] = 1
            K[j] = rng.uniform(0.01, 0.1) / N
        for p in rng.choice(ns, size=rng.integers(1, 4), replace=True):
            S[p, j] += 1
    lat = empty_lattice(X, Y, Z, slots, bytes_per_slot)
    occ = None
    total = int(density * N)
    per_sp = rng.multinomial(total, np.ones(ns) / ns)
    for s in range(ns):
        for st in range(nst):
            cnt = int(per_sp[s] // nst)
            if cnt:
                occ = place_particles(lat, sites, X, Y, Z, slots, bytes_per_slot, s + 1, cnt, st, rng, occ)
    return ModelSpec("random-%d" % seed, X, Y, Z, slots, bytes_per_slot, ns, nst, tau, spacing, rtype,
                     K, S, Dm, DF, RL, lat, sites, steps)


# --------------------------------------------------------------------------
# Config 3 (CME part): two-state gene expression, well mixed
# --------------------------------------------------------------------------

@dataclass
class CMESpec:
    """A well-mixed model as CMESolver::buildModel receives it
    (cme/CMESolver.h:200-201): reaction types, rate constants (one column),
    species-major stoichiometry S[NS, R] and dependency D[NS, R], initial
    counts."""
    name: str
    ns: int
    rtype: np.ndarray          # [R] uint32
    K: np.ndarray              # [R] float64
    S: np.ndarray              # [NS, R] int32
    D: np.ndarray              # [NS, R] uint32
    init: np.ndarray           # [NS] uint32
    max_time: float
    write_interval: float
    species_names: List[str] = field(default_factory=list)

    @property
    def nr(self):
        return int(len(self.rtype))


def two_state_gene(max_time=3600.0, write_interval=600.0):
    """The two-state gene model of lm::cme::TwoStateExpression
    (cme/TwoStateExpression.cpp:74-107): species gene-inactive, gene-active,
    mRNA, protein; reactions activation, inactivation, transcription (active
    gene -> + mRNA), translation (mRNA -> + protein), mRNA decay, protein
    decay, all first order.  Rates (per second) lie in 0.01..10: activation
    0.05, inactivation 0.2, transcription 2, translation 10, mRNA decay 0.5,
    protein decay 0.01.  One inactive gene, no mRNA or protein at t = 0."""
    S = np.array([[-1, 1, 0, 0, 0, 0],
                  [1, -1, 0, 0, 0, 0],
                  [0, 0, 1, 0, -1, 0],
                  [0, 0, 0, 1, 0, -1]], dtype=np.int32)
    D = np.array([[1, 0, 0, 0, 0, 0],
                  [0, 1, 1, 0, 0, 0],
                  [0, 0, 0, 1, 1, 0],
                  [0, 0, 0, 0, 0, 1]], dtype=np.uint32)
    rtype = np.full(6, FIRST, dtype=np.uint32)
    K = np.array([0.05, 0.2, 2.0, 10.0, 0.5, 0.01])
    init = np.array([1, 0, 0, 0], dtype=np.uint32)
    return CMESpec("two-state-gene", 4, rtype, K, S, D, init, max_time, write_interval,
                   ["gene_inactive", "gene_active", "mRNA", "protein"])


# --------------------------------------------------------------------------
# Config 4: serving stream of solve requests
# --------------------------------------------------------------------------

@dataclass
class ServeRequest:
    index: int
    arrival: float      # seconds after the stream starts
    edge: int
    ns: int
    density: float      # particles per site
    timesteps: int
    seed: int           # generator seed of the request's model and lattice


def serve_stream(seed=4, count=1000, rate=50.0, edges=tuple(range(16, 129, 8)), ns_range=(2, 50),
                 density_range=(0.5, 2.0), steps_range=(1000, 20000)):
    """A seeded Poisson arrival stream of solve requests: exponential
    inter-arrival times at `rate` per second, cubic lattice edge, species
    count, particle density and timestep count drawn uniformly."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=count))
    out = []
    for k in range(count):
        out.append(ServeRequest(
            index=k, arrival=float(t[k]), edge=int(rng.choice(edges)),
            ns=int(rng.integers(ns_range[0], ns_range[1] + 1)),
            density=float(rng.uniform(*density_range)),
            timesteps=int(rng.integers(steps_range[0], steps_range[1] + 1)),
            seed=int(rng.integers(1, 2 ** 31))))
    return out


def serve_problem(req, spacing=32e-9, tau=50e-6):
    """The model and lattice of one serving request: `req.ns` species with
    per-species D log-uniform in [1e-14, 5e-12] m^2/s, about one reaction per
    species (first order 0.1..10 /s, second order 1e5..1e7 /M/s, no two
    second-order reactions on the same pair), particles spread evenly over
    the species at `req.density` per site, one site type, ByteLattice 8."""
    rng = np.random.default_rng(req.seed)
    X = Y = Z = req.edge
    N = X * Y * Z
    ns, nst = req.ns, 1
    nr = ns
    DF = np.exp(rng.uniform(np.log(1e-14), np.log(5e-12), size=ns)).reshape(1, 1, ns)
    rtype = np.zeros(nr, dtype=np.uint32)
    K = np.zeros(nr)
    S = np.zeros((ns, nr), dtype=np.int32)
    Dm = np.zeros((ns, nr), dtype=np.uint32)
    pairs = set()
    for j in range(nr):
        if ns >= 2 and rng.random() < 0.5:
            while True:
                a, b = sorted(int(v) for v in rng.choice(ns, size=2, replace=False))
                if (a, b) not in pairs or len(pairs) >= ns * (ns - 1) // 2:
                    break
            if (a, b) in pairs:
                rtype[j] = FIRST
                K[j] = float(np.exp(rng.uniform(np.log(0.1), np.log(10.0))))
                S[a, j] -= 1
                Dm[a, j] = 1
            else:
                pairs.add((a, b))
                rtype[j] = SECOND
                K[j] = lm_rate(float(np.exp(rng.uniform(np.log(1e5), np.log(1e7)))), 2, spacing, N)
                S[a, j] -= 1
                S[b, j] -= 1
                Dm[a, j] = Dm[b, j] = 1
        else:
            a = int(rng.integers(ns))
            rtype[j] = FIRST
            K[j] = float(np.exp(rng.uniform(np.log(0.1), np.log(10.0))))
            S[a, j] -= 1
            Dm[a, j] = 1
        S[int(rng.integers(ns)), j] += 1
    RL = np.ones((nr, nst), dtype=np.uint32)
    lat = empty_lattice(X, Y, Z, 8, 1)
    sites = np.zeros(N, dtype=np.uint8)
    total = int(round(req.density * N))
    per = np.full(ns, total // ns)
    per[: total - per.sum()] += 1
    occ = None
    for sp in range(ns):
        if per[sp]:
            occ = place_particles(lat, sites, X, Y, Z, 8, 1, sp + 1, int(per[sp]), 0, rng, occ)
    return ModelSpec("serve-%d" % req.index, X, Y, Z, 8, 1, ns, nst, tau, spacing, rtype, K, S, Dm, DF, RL,
                     lat, sites, req.timesteps)


def batch_edges(seed=7, count=256, edges=(16, 24, 32, 48, 64)):
    rng = np.random.default_rng(seed)
    return [int(e) for e in rng.choice(edges, size=count)]
