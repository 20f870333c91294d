// Exception barrier for the C ABI: no C++ exception crosses an extern "C"
// entry; the message is stored for sundog_last_error() on this thread
// (src/capi_internal.h:46-56 has the same contract).
#pragma once

#include <exception>
#include <string>

namespace sdb {
void setError(const std::string& msg);
}

#define SDB_TRY try {
#define SDB_CATCH(errval)            \
  }                                  \
  catch (const std::exception& e) {  \
    ::sdb::setError(e.what());       \
    return errval;                   \
  }                                  \
  catch (...) {                      \
    ::sdb::setError("unknown error"); \
    return errval;                   \
  }
