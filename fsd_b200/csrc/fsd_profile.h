// Optional per-region device timing with CUDA events on the handle's stream.
// Regions nest freely; each records an event pair when profiling is on, and
// elapsed times are resolved when the caller reads them.
#pragma once

#include "fsd_internal.h"

namespace fsd {

enum Region {
    R_NLIST = 0,
    R_PRECOND_BUILD,
    R_SPREAD,
    R_FFT,
    R_GREEN,
    R_CONTRACT,
    R_REAL,
    R_RFU,
    R_PRECOND_APPLY,
    R_KRYLOV,
    R_LANCZOS,
    R_BROWNIAN_WAVE,
    R_LUB_OTHER,
    R_INTEGRATE,
    R_COUNT
};

void profile_begin(fsd_handle* h, int region);
void profile_end(fsd_handle* h, int region);
void profile_destroy(fsd_handle* h);

struct ProfRegion {
    fsd_handle* h;
    int r;
    ProfRegion(fsd_handle* h_, int r_) : h(h_), r(r_) { profile_begin(h, r); }
    ~ProfRegion() { profile_end(h, r); }
};

}  // namespace fsd
