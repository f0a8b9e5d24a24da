// pt_api_common.h — turning C++ failures into pt_status codes at the C boundary.
#pragma once

#include <exception>
#include <new>
#include <string>
#include "pt_host.h"

namespace ptb {
void set_last_error(const std::string &message);

// Runs `body`, mapping exceptions to a status and recording the message for pt_last_error().
template <class F> pt_status guard(F &&body) {
    try {
        body();
        return PT_OK;
    } catch(const Error &e) {
        set_last_error(e.what());
        return e.status;
    } catch(const std::bad_alloc &) {
        set_last_error("host allocation failed");
        return PT_INVALID_ARGUMENT;
    } catch(const std::exception &e) {
        set_last_error(e.what());
        return PT_INVALID_ARGUMENT;
    }
}
} // namespace ptb
