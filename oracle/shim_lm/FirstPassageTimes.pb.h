/* Stand-in for the generated lm::io::FirstPassageTimes message
 * (src/protobuf/FirstPassageTimes.proto). */
#ifndef LMB_SHIM_FIRSTPASSAGETIMES_PB_H
#define LMB_SHIM_FIRSTPASSAGETIMES_PB_H
#include <stdint.h>
#include <vector>
#include <google/protobuf/message.h>

namespace lm {
namespace io {

class FirstPassageTimes : public ::google::protobuf::Message {
public:
    void Clear() { species_ = 0; species_count_.clear(); first_passage_time_.clear(); }
    void set_species(int32_t s) { species_ = s; }
    int32_t species() const { return species_; }
    void add_species_count(int32_t c) { species_count_.push_back(c); }
    void add_first_passage_time(double t) { first_passage_time_.push_back(t); }
    int first_passage_time_size() const { return (int)first_passage_time_.size(); }

private:
    int32_t species_ = 0;
    std::vector<int32_t> species_count_;
    std::vector<double> first_passage_time_;
};

}  // namespace io
}  // namespace lm
#endif
