/* Lattice Microbes `.lm` trajectory file writer, C ABI.
 *
 * Writes the reference's `.lm` layout (docs/HDF5FileFormat.text;
 * io/SimulationFile.cpp, io/SimulationFile_create.cpp) as an HDF5 file that
 * libhdf5 and h5py read, without linking an HDF5 library: a 512-byte user
 * block starting "LMH5", superblock version 0, version-1 object headers,
 * symbol-table groups and version-1 B-trees, as libhdf5's default settings
 * write them.  Dataset names, types, shapes, chunking and gzip level follow
 * the reference:
 *
 *   /                       formatVersion = 4
 *   /Parameters             one string attribute per parameter
 *   /Model/Reaction         numberSpecies, numberReactions; InitialSpeciesCounts
 *                           u32[ns], ReactionTypes u32[nr], ReactionRateConstants
 *                           f64[nr][10], ReactionRateNoise f64[nr][2] (optional),
 *                           StoichiometricMatrix i32[ns][nr], DependencyMatrix
 *                           u32[ns][nr]                (SimulationFile.cpp:470-548)
 *   /Model/Diffusion        numberSpecies, numberReactions, numberSiteTypes,
 *                           latticeSpacing, lattice{X,Y,Z}Size, particlesPerSite,
 *                           bytes_per_particle; DiffusionMatrix f64[nst][nst][ns],
 *                           ReactionLocationMatrix u32[nr][nst], Lattice
 *                           u8|u32[X][Y][Z][P], LatticeSites u8[X][Y][Z]
 *                                                      (SimulationFile.cpp:690-870)
 *   /Simulations/%07d       SpeciesCounts i32[n][ns] and SpeciesCountTimes f64[n]
 *                           (chunks of 100 rows, extendable: SimulationFile.cpp:
 *                           2187-2226); LatticeTimes f64[n] + Lattice/%010d
 *                           u8|u32[X][Y][Z][P] (16^3 x P chunks, gzip 1:
 *                           SimulationFile.cpp:1166-1345); SiteTimes + Sites/%010d
 *                           u8[X][Y][Z] (SimulationFile.cpp:1347-1440);
 *                           MaxParticleCounts u32[ns+1], MaxSiteCounts u32[nst]
 *                           (MpdRdmeSolver.cu:921-932, SimulationFile.cpp:2368-2393)
 *
 * Lattice frames are written by a writer thread: the *_device calls transpose
 * the device lattice to [x][y][z][p] on the GPU (ByteLattice::
 * copyNativeToRowMajorByte order), copy it to pinned memory on the lattice's
 * stream and return; the thread compresses the 16^3 chunks in parallel and
 * appends them to the file, as the reference's DataOutputQueue +
 * LocalDataOutputWorker do (core/LocalDataOutputWorker.cpp:165-360).  Bulk
 * data goes to the end of the file as it arrives; the metadata (object
 * headers, B-trees, heaps) is written by lmb_lmfile_flush and
 * lmb_lmfile_close, after which the file on disk is complete.
 *
 * Every call returns LMB_OK or a negative status (lmb.h); LMB_E_IO for a
 * failed file operation.
 */
#ifndef LMB_LMFILE_H
#define LMB_LMFILE_H

#include <stdint.h>

#include "lmb.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct lmb_lmfile lmb_lmfile;

/* SimulationFile::create + open (SimulationFile_create.cpp:56-131): fails with
 * LMB_E_IO if the file exists.  The new file holds /Parameters, /Model and
 * /Simulations and formatVersion 4 and is complete on disk on return. */
int lmb_lmfile_create(const char *path, lmb_lmfile **out);

/* SimulationFile::setParameter (SimulationFile.cpp:322-336). */
int lmb_lmfile_set_parameter(lmb_lmfile *f, const char *key, const char *value);

/* SimulationFile::setReactionModel (SimulationFile.cpp:470-548):
 * rate_constants [nr][10] with unused columns NaN; noise [nr][2] (variance,
 * tau) or NULL for no noise table; S and D [ns][nr]. */
int lmb_lmfile_set_reaction_model(lmb_lmfile *f, uint32_t number_species, uint32_t number_reactions,
                                  const uint32_t *initial_counts, const uint32_t *types,
                                  const double *rate_constants, const double *noise, const int32_t *S,
                                  const uint32_t *D);

/* SimulationFile::setDiffusionModel (SimulationFile.cpp:690-760): DF
 * [nst][nst][ns], RL [nr][nst] (ignored when nr == 0). */
int lmb_lmfile_set_diffusion_model(lmb_lmfile *f, uint32_t number_species, uint32_t number_reactions,
                                   uint32_t number_site_types, double lattice_spacing, uint32_t X, uint32_t Y,
                                   uint32_t Z, uint32_t particles_per_site, uint32_t bytes_per_particle,
                                   const double *DF, const uint32_t *RL);

/* SimulationFile::setDiffusionModelLattice (SimulationFile.cpp:833-870):
 * row-major particles [X][Y][Z][P] (uint8 when bytes_per_particle is 1,
 * uint32 when 4) and site types [X][Y][Z]; sizes from the diffusion model. */
int lmb_lmfile_set_diffusion_model_lattice(lmb_lmfile *f, const void *particles, const uint8_t *sites);

/* SimulationFile::appendSpeciesCounts: `rows` rows of number_species counts
 * with their times. */
int lmb_lmfile_append_species_counts(lmb_lmfile *f, uint32_t replicate, uint32_t rows, uint32_t number_species,
                                     const double *times, const int32_t *counts);

/* SimulationFile::appendLattice / appendLattice_U32LE (SimulationFile.cpp:
 * 1166-1345) from a host row-major frame [X][Y][Z][P]; the data is copied
 * before the call returns. */
int lmb_lmfile_append_lattice(lmb_lmfile *f, uint32_t replicate, double time, uint32_t X, uint32_t Y, uint32_t Z,
                              uint32_t particles_per_site, uint32_t bytes_per_particle, const void *particles);

/* The same from a device lattice, asynchronously: transposed on the GPU and
 * copied to pinned memory in the lattice's stream order, then written by the
 * writer thread.  The lattice may be advanced again at once.  LMB_E_STATE
 * while an asynchronous run of the lattice is in flight. */
int lmb_lmfile_append_lattice_device(lmb_lmfile *f, uint32_t replicate, double time, lmb_lattice *lattice);

/* SimulationFile::appendSites (SimulationFile.cpp:1347-1440) from host site
 * types [X][Y][Z], or from the device lattice. */
int lmb_lmfile_append_sites(lmb_lmfile *f, uint32_t replicate, double time, uint32_t X, uint32_t Y, uint32_t Z,
                            const uint8_t *sites);
int lmb_lmfile_append_sites_device(lmb_lmfile *f, uint32_t replicate, double time, lmb_lattice *lattice);

/* MpdRdmeSolver::writeMaxCounts (MpdRdmeSolver.cu:921-932): MaxParticleCounts
 * and MaxSiteCounts of the replicate (each written once). */
int lmb_lmfile_write_max_counts(lmb_lmfile *f, uint32_t replicate, const uint32_t *max_particle_counts,
                                uint32_t n_particle, const uint32_t *max_site_counts, uint32_t n_site);

/* Element types of the generic calls below. */
#define LMB_H5_U8 1
#define LMB_H5_I8 2
#define LMB_H5_U16 3
#define LMB_H5_I16 4
#define LMB_H5_U32 5
#define LMB_H5_I32 6
#define LMB_H5_U64 7
#define LMB_H5_I64 8
#define LMB_H5_F32 9
#define LMB_H5_F64 10
#define LMB_H5_STRING 11 /* fixed-size, null-terminated ASCII */

/* Generic objects, for carrying an existing file's contents into a new one
 * (the runSolver path): a group (with its parents), an attribute on a group
 * or dataset (string_size: bytes per string including the terminator, for
 * LMB_H5_STRING; rank 0 is a scalar), and a dataset written now, contiguous
 * (chunk_dims NULL) or chunked (gzip_level -1 for none).  An extendable
 * dataset (first dimension unlimited; chunked) keeps its rows in memory so
 * that later appends (species counts, frame times) extend it. */
int lmb_lmfile_create_group(lmb_lmfile *f, const char *path);
int lmb_lmfile_set_attribute(lmb_lmfile *f, const char *path, const char *name, int type, uint32_t rank,
                             const uint64_t *dims, const void *data, uint32_t string_size);
int lmb_lmfile_write_dataset(lmb_lmfile *f, const char *group, const char *name, int type, uint32_t rank,
                             const uint64_t *dims, const uint64_t *chunk_dims, int gzip_level, int extendable,
                             const void *data);

/* Waits for the writer thread and writes the metadata: the file on disk is a
 * complete `.lm` file afterwards (the reference's checkpoint point,
 * SimulationFile.cpp:158-190). */
int lmb_lmfile_flush(lmb_lmfile *f);

/* SimulationFile::checkpoint (SimulationFile.cpp:158-190): flushes, then
 * copies the complete file to "<path>.chk" and writes that name (with its
 * terminator) to checkpoint_path when it fits in size bytes (else
 * LMB_E_ARG after the copy).  checkpoint_path may be NULL. */
int lmb_lmfile_checkpoint(lmb_lmfile *f, char *checkpoint_path, uint64_t size);

/* Frames written and bytes of compressed chunk data appended so far. */
int lmb_lmfile_stats(lmb_lmfile *f, uint64_t *frames, uint64_t *chunk_bytes);

/* Flushes, closes the file and frees the handle (also after an error). */
int lmb_lmfile_close(lmb_lmfile *f);

#ifdef __cplusplus
}
#endif

#endif
