// Definitions behind the opaque handles of include/sbe.h that more than one
// translation unit of the library needs.
#pragma once

#include <string>

#include "../../include/sbe.h"
#include "sbe_problem.h"

struct sbe_problem {
    sbe::Problem p;
    std::string unsupported;  // non-empty: valid input that this library does not build
};

namespace sbe {
// Records `msg` as the calling thread's sbe_last_error_message() and returns st.
sbe_status set_error(sbe_status st, const char *msg);
}  // namespace sbe
