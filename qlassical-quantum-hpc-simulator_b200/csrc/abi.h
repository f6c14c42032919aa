// abi.h -- the C ABI's error boundary: library errors (qlb::Error), host
// allocation failures and anything else thrown become a status code plus
// the thread's last-error message; nothing propagates across extern "C".
#pragma once

#include <new>
#include <stdexcept>
#include <string>

#include "engine.h"

namespace qlb {

template <typename F>
int guarded(F&& f) {
    try {
        f();
        return QLB_OK;
    } catch (const Error& err) {
        set_last_error(err.msg);
        return err.code;
    } catch (const std::bad_alloc&) {
        set_last_error("host allocation failed");
        return QLB_ERR_OOM;
    } catch (const std::exception& ex) {
        set_last_error(ex.what());
        return QLB_ERR_CUDA;
    } catch (...) {
        set_last_error("unknown error");
        return QLB_ERR_CUDA;
    }
}

inline void need(const void* p, const char* what) {
    if (!p) fail(QLB_ERR_INVALID_ARG, std::string(what) + " is null");
}

}  // namespace qlb
