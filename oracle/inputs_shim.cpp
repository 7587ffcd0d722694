// inputs_shim.cpp -- TEST INFRASTRUCTURE ONLY. The error plumbing that the
// synthetic-input builder (qublar_b200/csrc/qb_synth.cpp) needs when it is
// compiled on its own, host code only, into oracle/libqb_inputs.so: the
// reference arm of bench.py and the CPU-baseline legs build their inputs
// with it without loading the solver library. Same messages, no CUDA.
#include <string>

#include "qb_internal.hpp"

namespace qb {

namespace {
thread_local std::string g_last_error;
}

void set_error(const std::string& msg) { g_last_error = msg; }

qb_status fail(qb_status s, const std::string& msg) {
    g_last_error = msg;
    return s;
}

}  // namespace qb

extern "C" const char* qb_last_error(void) { return qb::g_last_error.c_str(); }
