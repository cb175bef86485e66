/*
 * Stand-in for protobuf's Message base class, for building the reference's
 * CPU solvers (NextSubvolumeSolver, GillespieDSolver) without libprotobuf.
 * Test infrastructure only: the reference code uses messages as plain
 * containers handed to the output queue.
 */
#ifndef LMB_SHIM_PROTOBUF_MESSAGE_H
#define LMB_SHIM_PROTOBUF_MESSAGE_H
#include <cassert>  /* real protobuf headers bring this in; RDMESolver.cpp relies on it */
#include <cstddef>
#include <string>
#include <vector>

namespace google {
namespace protobuf {

class Message {
public:
    virtual ~Message() {}
};

/* The part of RepeatedField the reference reads: data() and size(). */
template <typename T>
class RepeatedField {
public:
    const T *data() const { return v.empty() ? nullptr : v.data(); }
    int size() const { return (int)v.size(); }
    std::vector<T> v;
};

}  // namespace protobuf
}  // namespace google
#endif
