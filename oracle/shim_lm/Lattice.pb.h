/* Stand-in for the generated lm::io::Lattice frame header message
 * (src/protobuf/Lattice.proto). */
#ifndef LMB_SHIM_LATTICE_PB_H
#define LMB_SHIM_LATTICE_PB_H
#include <stdint.h>
#include <google/protobuf/message.h>

namespace lm {
namespace io {

class Lattice : public ::google::protobuf::Message {
public:
    void Clear() { x_ = y_ = z_ = p_ = 0; time_ = 0.0; }
    void set_lattice_x_size(uint32_t v) { x_ = v; }
    void set_lattice_y_size(uint32_t v) { y_ = v; }
    void set_lattice_z_size(uint32_t v) { z_ = v; }
    void set_particles_per_site(uint32_t v) { p_ = v; }
    void set_time(double t) { time_ = t; }

private:
    uint32_t x_ = 0, y_ = 0, z_ = 0, p_ = 0;
    double time_ = 0.0;
};

}  // namespace io
}  // namespace lm
#endif
