// Status-code plumbing for the C ABI: no exception or exit crosses it.
#pragma once

#include <exception>
#include <new>
#include <string>

#include "blest.h"
#include "common.hpp"

namespace blest {

void set_last_error(const std::string& msg);

inline void require(bool ok, const char* msg) {
    if (!ok) throw Error(BLEST_ERR_INVALID_ARG, msg);
}

template <class F>
int guarded(F&& f) {
    try {
        f();
        return BLEST_OK;
    } catch (const Error& e) {
        set_last_error(e.what());
        return e.code;
    } catch (const std::bad_alloc&) {
        set_last_error("host allocation failed");
        return BLEST_ERR_OOM;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return BLEST_ERR_INVALID_ARG;
    } catch (...) {
        set_last_error("unknown error");
        return BLEST_ERR_INVALID_ARG;
    }
}

}  // namespace blest
