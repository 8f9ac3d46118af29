// Error type and status codes of the host runtime. Errors never cross the
// C ABI as exceptions: each entry point converts them to a ZX_E* status and a
// thread-local message (see include/zindex.h).
#pragma once
#include <stdexcept>
#include <string>

namespace zx {

enum Status : int {
  kOk = 0,
  kEInval = 1,    // invalid argument
  kEFormat = 2,   // malformed index, manifest or query file
  kEIo = 3,       // file system error
  kENoMem = 4,    // device or host memory exhausted / admission refused
  kECuda = 5,     // CUDA runtime error
  kETimeout = 6,  // a bounded device wait expired
  kEUnsupported = 7,
};

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] inline void raise(int code, const std::string& msg) { throw Error(code, msg); }
inline void check(bool ok, int code, const char* msg) {
  if (!ok) throw Error(code, msg);
}
inline void check_format(bool ok, const char* msg) {
  if (!ok) throw Error(kEFormat, msg);
}

}  // namespace zx
