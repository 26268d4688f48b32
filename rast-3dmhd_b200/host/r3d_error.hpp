// r3d_error.hpp - per-thread error message behind r3d_last_error() and the status-code guard
// used by every C entry point (the reference exits the process instead, src/gpu.cpp:117-139).
#pragma once

#include <exception>
#include <new>
#include <stdexcept>
#include <string>

#include "r3d_gpu.h"

namespace r3db {

void set_error(const std::string& msg);
void clear_error();

// Error carrying an r3d status code.
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

// Run f(); map exceptions to status codes and record the message.
template <class F>
int guarded(F&& f) {
    try {
        clear_error();
        f();
        return R3D_OK;
    } catch (const Error& e) {
        set_error(e.what());
        return e.code;
    } catch (const std::invalid_argument& e) {
        set_error(e.what());
        return R3D_EINVAL;
    } catch (const std::bad_alloc&) {
        set_error("host allocation failed");
        return R3D_ENOMEM;
    } catch (const std::exception& e) {
        set_error(e.what());
        return R3D_EINVAL;
    }
}

}  // namespace r3db
