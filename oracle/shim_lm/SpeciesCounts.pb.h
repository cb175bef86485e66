/* Stand-in for the generated lm::io::SpeciesCounts message (src/protobuf/
 * SpeciesCounts.proto): a time column and a row of counts per entry. */
#ifndef LMB_SHIM_SPECIESCOUNTS_PB_H
#define LMB_SHIM_SPECIESCOUNTS_PB_H
#include <stdint.h>
#include <chrono>
#include <vector>
#include <google/protobuf/message.h>

namespace lm {
namespace io {

/* Wall-clock second (steady clock) at which each record's time entry was
 * added on this thread: the solver adds one per record as its simulated time
 * crosses a write time, so the stamps time stretches of one trajectory with
 * the solver's set-up before the first one. */
inline std::vector<double> &record_walls()
{
    static thread_local std::vector<double> walls;
    return walls;
}

class SpeciesCounts : public ::google::protobuf::Message {
public:
    void Clear() { number_species_ = 0; number_entries_ = 0; time_.clear(); species_count_.clear(); }
    void set_number_species(int32_t n) { number_species_ = n; }
    int32_t number_species() const { return number_species_; }
    void set_number_entries(int32_t n) { number_entries_ = n; }
    int32_t number_entries() const { return number_entries_; }
    void add_time(double t)
    {
        time_.push_back(t);
        record_walls().push_back(
            std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count());
    }
    int time_size() const { return (int)time_.size(); }
    double time(int i) const { return time_[i]; }
    void add_species_count(int32_t c) { species_count_.push_back(c); }
    int species_count_size() const { return (int)species_count_.size(); }
    int32_t species_count(int i) const { return species_count_[i]; }

private:
    int32_t number_species_ = 0;
    int32_t number_entries_ = 0;
    std::vector<double> time_;
    std::vector<int32_t> species_count_;
};

}  // namespace io
}  // namespace lm
#endif
