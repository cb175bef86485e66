"""B200-native MPD-RDME solver for Lattice Microbes models.

The solver runs in liblmb200.so (CUDA for sm_100a behind the C ABI in
include/lmb.h).  ``solver`` is the Python face of that ABI (contexts, models,
lattices, batches, the solve server, CME ensembles); ``rdme`` gives the
MpdRdmeSolver / IntMpdRdmeSolver classes pyLM and jLM scripts subclass, and
runSolver on `.lm` files; ``lmfile`` reads and writes `.lm` (HDF5) files
without an HDF5 library (the writer is include/lmb_lmfile.h in the same
library); ``replicas`` runs one replicate per GPU under torch.distributed;
``configs`` generates seeded synthetic problems.  Importing ``solver`` fails when the
library has not been built: there is no CPU fallback.
"""
__all__ = ["configs", "lmfile", "rdme", "replicas", "solver"]
