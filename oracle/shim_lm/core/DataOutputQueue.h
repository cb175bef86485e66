/*
 * Stand-in for lm::main::DataOutputQueue (src/core/DataOutputQueue.h:57-125)
 * for the reference CPU solver build: instead of serialising data sets for
 * the HDF5 writer thread, the queue of the calling thread keeps the species
 * counts the solver pushes, so the harness can hand them back.  The message
 * type constants keep the reference's values.
 */
#ifndef LMB_SHIM_DATAOUTPUTQUEUE_H
#define LMB_SHIM_DATAOUTPUTQUEUE_H
#include <cstddef>
#include <vector>
#include <google/protobuf/message.h>
#include "core/Types.h"
#include "core/Exceptions.h"
#include "core/Print.h"

namespace lm {
namespace main {

class DataOutputQueue {
public:
    static const uint SPECIES_COUNTS = 10;
    static const uint FIRST_PASSAGE_TIMES = 11;
    static const uint PARAMETER_VALUES = 12;
    static const uint BYTE_LATTICE = 20;
    static const uint INT_LATTICE = 21;
    static const uint SITE_LATTICE = 22;

    /* One queue per thread: replicates run on separate threads. */
    static DataOutputQueue *getInstance();

    void pushDataSet(uint type, uint replicate, ::google::protobuf::Message *message, void *payload = NULL,
                     size_t payloadSize = 0, void (*payloadSerializer)(void *, void *, size_t) = NULL);

    /* Captured species counts: times[e], counts[e * numberSpecies + s]. */
    std::vector<double> times;
    std::vector<uint32_t> counts;
    uint numberSpecies = 0;
    uint latticeFrames = 0;
};

}  // namespace main
}  // namespace lm
#endif
