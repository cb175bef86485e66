/* Stand-in for the generated lm::io::ReactionModel message
 * (src/protobuf/ReactionModel.proto), with the accessors that
 * CMESolver::setReactionModel reads. */
#ifndef LMB_SHIM_REACTIONMODEL_PB_H
#define LMB_SHIM_REACTIONMODEL_PB_H
#include <stdint.h>
#include <vector>
#include <google/protobuf/message.h>

namespace lm {
namespace io {

class ReactionModel_Reaction {
public:
    uint32_t type() const { return type_; }
    int rate_constant_size() const { return (int)rate_constant_.size(); }
    double rate_constant(int i) const { return rate_constant_[i]; }
    uint32_t type_ = 0;
    std::vector<double> rate_constant_;
};

class ReactionModel : public ::google::protobuf::Message {
public:
    uint32_t number_species() const { return number_species_; }
    uint32_t number_reactions() const { return number_reactions_; }
    int reaction_size() const { return (int)reaction_.size(); }
    const ReactionModel_Reaction &reaction(int i) const { return reaction_[i]; }
    const ::google::protobuf::RepeatedField<uint32_t> &initial_species_count() const { return initial_species_count_; }
    const ::google::protobuf::RepeatedField<int32_t> &stoichiometric_matrix() const { return stoichiometric_matrix_; }
    const ::google::protobuf::RepeatedField<uint32_t> &dependency_matrix() const { return dependency_matrix_; }

    uint32_t number_species_ = 0, number_reactions_ = 0;
    std::vector<ReactionModel_Reaction> reaction_;
    ::google::protobuf::RepeatedField<uint32_t> initial_species_count_;
    ::google::protobuf::RepeatedField<int32_t> stoichiometric_matrix_;
    ::google::protobuf::RepeatedField<uint32_t> dependency_matrix_;
};

}  // namespace io
}  // namespace lm
#endif
