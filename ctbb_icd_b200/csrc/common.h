// Internal helpers shared by the host and device translation units.
#pragma once

#include <stdarg.h>
#include <stdio.h>

#include <string>

#include "../../include/ctbb_icd_b200.h"

namespace ctbb {

// Thread-local last-error message behind ctbb_last_error().
void set_error(const char* fmt, ...);
void clear_error();

// Returns `st` after recording a formatted message.
ctbb_status fail(ctbb_status st, const char* fmt, ...);

inline int n_ffs(const ctbb_geom_c& g) {
    // setup.cpp:202 — 2^Zffs * 2^Phiffs focal spots per stack
    return (int)((1ull << g.Zffs) * (1ull << g.Phiffs));
}

}  // namespace ctbb
