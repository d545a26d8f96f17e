// The C-ABI's error boundary: each entry point runs its body through guarded(), which turns a library error
// into its status code (a std::exception of another kind into B200_STATUS_INVALID_ARGUMENT) and keeps the
// message for b200_last_error(); a call that succeeds clears the message.
#pragma once
#include <exception>

#include "../../include/abacus_b200.h"
#include "common.h"

namespace b200 {

template <typename F> int guarded(F&& f) {
    try {
        f();
        set_last_error("");
        return B200_STATUS_OK;
    } catch (const Error& e) {
        set_last_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return B200_STATUS_INVALID_ARGUMENT;
    }
}

}  // namespace b200
