/* Stand-in for the generated lm::io::ParameterValues message
 * (src/protobuf/ParameterValues.proto). */
#ifndef LMB_SHIM_PARAMETERVALUES_PB_H
#define LMB_SHIM_PARAMETERVALUES_PB_H
#include <string>
#include <vector>
#include <google/protobuf/message.h>

namespace lm {
namespace io {

class ParameterValues : public ::google::protobuf::Message {
public:
    void Clear() { parameter_.clear(); time_.clear(); value_.clear(); }
    void set_parameter(const std::string &p) { parameter_ = p; }
    void add_time(double t) { time_.push_back(t); }
    void add_value(double v) { value_.push_back(v); }
    int value_size() const { return (int)value_.size(); }

private:
    std::string parameter_;
    std::vector<double> time_;
    std::vector<double> value_;
};

}  // namespace io
}  // namespace lm
#endif
