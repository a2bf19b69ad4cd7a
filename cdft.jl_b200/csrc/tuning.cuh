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
    // The two sections reduce in different orders, and on a few isotherm state points the
    // evaluation count is chaotic in the last bits, so the batch time mixes the section's cost
    // with which evaluation count a state point happens to land on.  The sweep therefore
    // compares the time per evaluation of the critical path (batch time / the largest
    // evaluation count), and per-stage clock64 timers agree: the Anderson section costs
    // 2.65 us (block) vs 4.41 us (warp) per evaluation at N = 186 and 1.7 vs 3.6 us at N = 400,
    // so 0 (the whole block for every system).
    int pers_warp_aa_max_elem = 0;
    // persistent engine: two CTAs per system (a cluster of two splitting the convolution tasks
    // and the Phi points, distributed shared memory between them) when the batch fits the
    // device in one wave of pairs; same arithmetic, so the same results as one CTA per system
    int pers_cluster = 1;
    // 3D grids: the strided y and z FFT passes as persistent TMA tile kernels (1) or as one
    // block per tile with per-thread loads (0); both compute the same arithmetic
    int fft3d_tma = 1;
    // 3D grids: the inverse x pass of the 8 convolved fields, Phi and the forward x pass in one
    // kernel (1) or three (0); both compute the same arithmetic.  Measured at 128^3 and 256^3
    // (FP64 and mixed): the three kernels are faster (the fused block holds 9 fields of its
    // rows and runs one block per SM), so 0.
    int fft3d_fused_phi = 0;
    // radial grids: the dense weighted-density operators of a batch as FP64 tensor-core GEMMs
    // over column tiles of systems that share one operator, 8 rows per CTA (1) or 16 rows per
    // CTA sharing the input fragments (2, the same bits as 1), or one warp-per-row FFMA
    // matrix-vector launch per system (0).  The GEMM and the FFMA kernel sum in different
    // orders; the GEMM's per-element sum does not depend on the other systems of the tile.
    // Measured on the spherical-pore isotherm batch: dense stage 274.5 us (0), 12.35 us (1),
    // 10.30 us (2), so 2.
    int radial_dmma = 2;
};

static TunedShapes g_tuned;

struct TunedEntry {
    const char* name;
    int TunedShapes::*field;
    int lo, hi;
};

static const TunedEntry kTunedEntries[] = {
    {"pers_warp_aa_max_elem", &TunedShapes::pers_warp_aa_max_elem, 0, 1 << 30},
    {"pers_cluster", &TunedShapes::pers_cluster, 0, 1},
    {"fft3d_tma", &TunedShapes::fft3d_tma, 0, 1},
    {"fft3d_fused_phi", &TunedShapes::fft3d_fused_phi, 0, 1},
    {"radial_dmma", &TunedShapes::radial_dmma, 0, 2},
};

inline const TunedEntry* tuned_entry(const char* name)
{
    if (!name) return nullptr;
    for (const TunedEntry& e : kTunedEntries)
        if (std::strcmp(e.name, name) == 0) return &e;
    return nullptr;
}
