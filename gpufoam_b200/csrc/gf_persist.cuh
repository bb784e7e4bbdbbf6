// The persistent work-queue solve kernel (sm_100a), shared by the per-G
// instantiation files gf_persist_g*.cu (one translation unit per group size,
// so that the variants compile in parallel).
//
// CTAs sized to the SMs; groups of G threads pull cells from an atomic work
// queue until it is empty. G <= 32: several groups per CTA (at most 128
// threads); G = 64, 128, 256: one group (one cell at a time) per CTA. The
// per-cell workspace lives in shared memory (SHARED) or in an HBM slot per
// resident group. Mixed mechanisms are selected by the per-cell id.
#pragma once

#include <cuda_runtime.h>

#include "gf_device.cuh"
#include "gf_internal.h"

namespace gf {

constexpr int kMaxMechs = 4;


struct MechSet {
    DevMech m[kMaxMechs];
    int n;
};

// The cell's mechanism, or null for an id outside the solver's mechanisms: the
// cell is then not integrated, its status says so, and it counts as failed.
__device__ __forceinline__ const DevMech* pick(const MechSet& P, const LaunchArgs& a, long long cell) {
    const int id = a.mech_id ? a.mech_id[cell] : 0;
    return (id >= 0 && id < P.n) ? &P.m[id] : nullptr;
}

// Such a cell leaves the solve unchanged: its output row is a copy of its
// input row (the whole row stride), its RR row is zero, its counters are zero
// and its deltaTChem is left as it was; it is left out of the min over cells.
template <int G>
__device__ __forceinline__ void reject_cell(const Grp<G>& g, const LaunchArgs& a, long long cell) {
    if (a.Ynew) {
        const double* yi = a.Y0 + (size_t)cell * a.ld_y;
        double* yo = a.Ynew + (size_t)cell * a.ld_y;
        for (int i = g.lane; i < a.ld_y; i += G) yo[i] = yi[i];
    }
    if (a.RR)
        for (int i = g.lane; i < a.ld_rr; i += G) a.RR[(size_t)cell * a.ld_rr + i] = 0.0;
    if (g.lane == 0) {
        if (a.status) a.status[cell] = GF_CELL_BAD_MECHANISM;
        if (a.counters) {
            a.counters[2 * cell] = 0;
            a.counters[2 * cell + 1] = 0;
        }
        atomicAdd(a.queue + 4, 1ull);
    }
}

// Registers per thread the kernel is compiled for: SLIM = 1, at most 128
// (512 resident threads per SM); otherwise up to 255, except for 64 threads
// per cell, capped at 200 so that five 64-thread CTAs fit an SM's registers
// (their workspaces fit its shared memory: 45 KB each at 53 species).
template <int G>
struct PersistShape {
    static constexpr int max_regs(int slim) { return slim ? 128 : (G == 64 ? 200 : 255); }
};

// NB: columns per LU panel; MS > 0: the matrix size m of every mechanism of
// the launch, fixed at compile time (process_cell).
template <int G, bool SHARED, int SLIM, int NB = 8, int MS = 0>
__global__ void __maxnreg__(PersistShape<G>::max_regs(SLIM))
    persistent_kernel(const MechSet P, const LaunchArgs a, int ws_per_cell, long long n_slots) {
    extern __shared__ double smem[];
    Grp<G> g;
    const int gpb = G > 32 ? 1 : blockDim.x / G;
    const int gib = G > 32 ? 0 : threadIdx.x / G;
    const long long slot = (long long)blockIdx.x * gpb + gib;
    for (;;) {
        long long cell = 0;
        if (g.lane == 0) cell = (long long)atomicAdd(a.queue, 1ull);
        cell = g.bcast_ll(cell, 0);
        if (cell >= a.n_cells) break;
        const DevMech* Mp = pick(P, a, cell);
        if (!Mp) {
            reject_cell(g, a, cell);
            continue;
        }
        const DevMech& M = *Mp;
        if (SHARED) {
            process_cell<G, WsC, false, NB, MS>(g, M, WsC{smem + (size_t)gib * ws_per_cell}, a, (int)cell);
        } else if (G == 1) {
            process_cell<G, WsS, false, NB, MS>(g, M, WsS{a.ws + slot, n_slots}, a, (int)cell);
        } else {
            process_cell<G, WsC, false, NB, MS>(g, M, WsC{a.ws + slot * ws_per_cell}, a, (int)cell);
        }
    }
}

template <int G, int NB = 8, int MS = 0>
const void* persistent_variant(bool shared, int slim) {
    if (shared)
        return slim ? reinterpret_cast<const void*>(&persistent_kernel<G, true, 1, NB, MS>)
                    : reinterpret_cast<const void*>(&persistent_kernel<G, true, 0, NB, MS>);
    return slim ? reinterpret_cast<const void*>(&persistent_kernel<G, false, 1, NB, MS>)
                : reinterpret_cast<const void*>(&persistent_kernel<G, false, 0, NB, MS>);
}

// The tuned variants of the 32-, 64-, 96- and 128-thread forms (gf_persist_g<G>_tuned.cu):
// LU panels of 4 or 16 columns (workspace in shared memory), and the matrix
// size fixed at compile time for the 10-, 53- and 100-species mechanisms
// (m = 11, 54, 101; workspace in shared memory or HBM; for m = 54 also with
// 4-column panels). Each with the register budget the form is usually run with
// (SLIM for 96 and 128 threads); nullptr for a variant that is not compiled.
constexpr int kTunedSlim(int G) { return (G == 128 || G == 96) ? 1 : 0; }
template <int G, int S, int NB, int MS>
const void* tuned_kernel(bool shared) {
    return shared ? reinterpret_cast<const void*>(&persistent_kernel<G, true, S, NB, MS>)
                  : reinterpret_cast<const void*>(&persistent_kernel<G, false, S, NB, MS>);
}
template <int G>
const void* persistent_tuned_variant(bool shared, int slim, int nb, int ms) {
    if (slim != kTunedSlim(G)) return nullptr;
    constexpr int S = kTunedSlim(G);
    if (ms == 0) {
        if (!shared) return nullptr;
        if (nb == 4) return tuned_kernel<G, S, 4, 0>(true);
        if (nb == 16) return tuned_kernel<G, S, 16, 0>(true);
        return nullptr;
    }
    if (ms == 54) {
        if (nb == 4) return tuned_kernel<G, S, 4, 54>(shared);
        if (nb == 8) return tuned_kernel<G, S, 8, 54>(shared);
        return nullptr;
    }
    if (nb != 8) return nullptr;
    if (ms == 11) return tuned_kernel<G, S, 8, 11>(shared);
    if (ms == 101) return tuned_kernel<G, S, 8, 101>(shared);
    return nullptr;
}

// defined in gf_persist_g<G>.cu
const void* persistent_fn_g1(bool shared, int slim);
const void* persistent_fn_g2(bool shared, int slim);
const void* persistent_fn_g4(bool shared, int slim);
const void* persistent_fn_g8(bool shared, int slim);
const void* persistent_fn_g16(bool shared, int slim);
const void* persistent_fn_g32(bool shared, int slim);
const void* persistent_fn_g64(bool shared, int slim);
const void* persistent_fn_g96(bool shared, int slim);
const void* persistent_fn_g128(bool shared, int slim);
const void* persistent_fn_g256(bool shared, int slim);
// defined in gf_persist_g<G>_tuned.cu
const void* persistent_tuned_fn_g32(bool shared, int slim, int nb, int ms);
const void* persistent_tuned_fn_g64(bool shared, int slim, int nb, int ms);
const void* persistent_tuned_fn_g96(bool shared, int slim, int nb, int ms);
const void* persistent_tuned_fn_g128(bool shared, int slim, int nb, int ms);

#ifdef GF_PHASE_TIMERS
// phase-timer accumulators of the gf_persist_g<G>.cu units (profiling builds)
int phase_cycles_g1(unsigned long long* out, int reset);
int phase_cycles_g2(unsigned long long* out, int reset);
int phase_cycles_g4(unsigned long long* out, int reset);
int phase_cycles_g8(unsigned long long* out, int reset);
int phase_cycles_g16(unsigned long long* out, int reset);
int phase_cycles_g32(unsigned long long* out, int reset);
int phase_cycles_g64(unsigned long long* out, int reset);
int phase_cycles_g96(unsigned long long* out, int reset);
int phase_cycles_g128(unsigned long long* out, int reset);
int phase_cycles_g256(unsigned long long* out, int reset);
int phase_cycles_adj(unsigned long long* out, int reset);
// the tuned variants' units (gf_persist_g<G>_tuned.cu)
int phase_cycles_g32t(unsigned long long* out, int reset);
int phase_cycles_g64t(unsigned long long* out, int reset);
int phase_cycles_g96t(unsigned long long* out, int reset);
int phase_cycles_g128t(unsigned long long* out, int reset);
#endif

}  // namespace gf
