// Internal host-side helpers shared by the C++ translation units.
#pragma once

#include <exception>
#include <string>
#include <utility>

#include "capacmd.h"

namespace capac {

// Failure carried to the C ABI as (status, message).
struct Error : std::exception {
    int code;
    std::string msg;
    Error(int c, std::string m) : code(c), msg(std::move(m)) {}
    const char *what() const noexcept override { return msg.c_str(); }
};

void set_last_error(const std::string &msg);

// Run f, turning exceptions into a status code and the thread's last error.
template <class F>
int guard(F &&f)
{
    try {
        f();
        return CAPAC_OK;
    } catch (const Error &e) {
        set_last_error(e.msg);
        return e.code;
    } catch (const std::exception &e) {
        set_last_error(e.what());
        return CAPAC_ERR_INVALID;
    } catch (...) {
        set_last_error("unknown error");
        return CAPAC_ERR_INVALID;
    }
}

capac_desc *desc_load(const char *gro, const char *par, const char *mds);
void desc_free(capac_desc *d);
void derive(const capac_desc *d, capac_consts *c);

}  // namespace capac
