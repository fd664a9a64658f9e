// Embeds the tabulated near-field resistance functions (92,000 bytes:
// float32 dist[1000] then vals[1000][22]) extracted from the reference's
// Stokes_ResistanceTable.cc by fsd_b200/data/extract_resistance_table.py.
#include "fsd_internal.h"

#ifndef FSD_RESTABLE_PATH
#error "FSD_RESTABLE_PATH must name fsd_b200/data/resistance_table.bin"
#endif

__asm__(
    ".section .rodata\n"
    ".balign 16\n"
    ".local fsd_restable_blob\n"
    "fsd_restable_blob:\n"
    ".incbin \"" FSD_RESTABLE_PATH "\"\n"
    ".previous\n");

extern "C" const float fsd_restable_blob[];

namespace fsd {
const float* resistance_table_dist() { return fsd_restable_blob; }
const float* resistance_table_vals() { return fsd_restable_blob + kResRows; }
}  // namespace fsd
