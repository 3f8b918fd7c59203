// Status codes and the exception that carries one to the C ABI boundary, plus the per-thread
// last-error slot (include/spektralab.h: "message in the thread's last-error slot").
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>

#include "spektralab.h"

namespace spkb {

class Error : public std::runtime_error {
public:
    Error(int32_t status, const std::string& msg) : std::runtime_error(msg), status_(status) {}
    int32_t status() const { return status_; }

private:
    int32_t status_;
};

[[noreturn]] inline void fail(int32_t status, const std::string& msg) { throw Error(status, msg); }
[[noreturn]] inline void fail_user(const std::string& msg) { fail(SPK_ERR_USER, msg); }
[[noreturn]] inline void fail_gpu(const std::string& msg) { fail(SPK_ERR_GPU, msg); }
[[noreturn]] inline void fail_io(const std::string& msg) { fail(SPK_ERR_IO, msg); }
[[noreturn]] inline void fail_internal(const std::string& msg) { fail(SPK_ERR_INTERNAL, msg); }
[[noreturn]] inline void fail_invalid(const std::string& msg) { fail(SPK_ERR_INVALID_ARG, msg); }
[[noreturn]] inline void fail_unsupported(const std::string& msg) { fail(SPK_ERR_UNSUPPORTED, msg); }
[[noreturn]] inline void fail_cancelled() { fail(SPK_ERR_CANCELLED, "render cancelled"); }

namespace last_error {
void set(const std::string& msg);
void clear();
const char* get();
}  // namespace last_error

}  // namespace spkb
