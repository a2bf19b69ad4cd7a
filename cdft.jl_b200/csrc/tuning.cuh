// Launch shapes chosen by the project's autotuner (cdft.jl_b200/tune.py).
//
// Every entry changes how work is mapped onto the B200, never which arithmetic a
// system sees for a given problem: entries that could move a reduction order are
// per-system rules (a threshold on the system's own size), so a system converged
// alone or inside a batch still gets bit-identical results.  The defaults are the
// values the sweep measured on B200; cdft_tuning_set overrides one for the process
// (the sweep itself uses it).
#pragma once
#include <cstring>

struct TunedShapes {
    // persistent engine: a system of at most this many elements (N * nc) runs the Anderson
    // vector slots on one warp (no block barriers); larger systems use the whole block.
    // Measured on the 64-point isotherm (N = 100..400, m = 5, three-pass Anderson update):
    // 11.26 ms per batch with 0, 10.74 with 256, 10.67 with 512, 10.66 with 1024, so 1024
    // (every isotherm system takes the warp path).
    int pers_warp_aa_max_elem = 1024;
    // 3D grids: the strided y and z FFT passes as persistent TMA tile kernels (1) or as one
    // block per tile with per-thread loads (0); both compute the same arithmetic
    int fft3d_tma = 1;
    // 3D grids: the inverse x pass of the 8 convolved fields, Phi and the forward x pass in one
    // kernel (1) or three (0); both compute the same arithmetic.  Measured at 128^3 and 256^3
    // (FP64 and mixed): the three kernels are faster (the fused block holds 9 fields of its
    // rows and runs one block per SM), so 0.
    int fft3d_fused_phi = 0;
};

static TunedShapes g_tuned;

struct TunedEntry {
    const char* name;
    int TunedShapes::*field;
    int lo, hi;
};

static const TunedEntry kTunedEntries[] = {
    {"pers_warp_aa_max_elem", &TunedShapes::pers_warp_aa_max_elem, 0, 1 << 30},
    {"fft3d_tma", &TunedShapes::fft3d_tma, 0, 1},
    {"fft3d_fused_phi", &TunedShapes::fft3d_fused_phi, 0, 1},
};

inline const TunedEntry* tuned_entry(const char* name)
{
    if (!name) return nullptr;
    for (const TunedEntry& e : kTunedEntries)
        if (std::strcmp(e.name, name) == 0) return &e;
    return nullptr;
}
