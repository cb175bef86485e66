/* Stand-in for the generated lm::io::DiffusionModel message
 * (src/protobuf/DiffusionModel.proto), with the accessors that
 * RDMESolver::setDiffusionModel reads. */
#ifndef LMB_SHIM_DIFFUSIONMODEL_PB_H
#define LMB_SHIM_DIFFUSIONMODEL_PB_H
#include <stdint.h>
#include <google/protobuf/message.h>

namespace lm {
namespace io {

class DiffusionModel : public ::google::protobuf::Message {
public:
    uint32_t number_species() const { return number_species_; }
    uint32_t number_reactions() const { return number_reactions_; }
    uint32_t number_site_types() const { return number_site_types_; }
    int diffusion_matrix_size() const { return diffusion_matrix_.size(); }
    const ::google::protobuf::RepeatedField<double> &diffusion_matrix() const { return diffusion_matrix_; }
    const ::google::protobuf::RepeatedField<uint32_t> &reaction_location_matrix() const { return reaction_location_matrix_; }
    uint32_t lattice_x_size() const { return x_; }
    uint32_t lattice_y_size() const { return y_; }
    uint32_t lattice_z_size() const { return z_; }
    uint32_t particles_per_site() const { return p_; }
    uint32_t bytes_per_particle() const { return b_; }
    double lattice_spacing() const { return spacing_; }

    uint32_t number_species_ = 0, number_reactions_ = 0, number_site_types_ = 0;
    ::google::protobuf::RepeatedField<double> diffusion_matrix_;
    ::google::protobuf::RepeatedField<uint32_t> reaction_location_matrix_;
    uint32_t x_ = 0, y_ = 0, z_ = 0, p_ = 0, b_ = 1;
    double spacing_ = 0.0;
};

}  // namespace io
}  // namespace lm
#endif
