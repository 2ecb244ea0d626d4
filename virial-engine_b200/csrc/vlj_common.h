// Host-side helpers shared by the C ABI sources.
#pragma once

#include "virial_lj.h"

namespace vlj {

// Records a message for vlj_last_error() and returns `s`.
vlj_status fail(vlj_status s, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
void clear_error();

}  // namespace vlj
