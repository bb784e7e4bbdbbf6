// Kernels and launchers of the per-cell chemistry path (sm_100a).
//
//  * plain_kernel      — one thread per cell, one launch over all cells, per-cell
//                        scratch interleaved in HBM: the reference's launch model
//                        (for_each_index.H:25-48, singleCellSolver.H:27-51) with
//                        coalesced scratch.
//  * persistent_kernel — gf_persist.cuh (instantiated in gf_persist_g*.cu): one
//                        CTA set sized to the SMs; groups of G threads (1..256)
//                        pull cells from an atomic work queue, scratch in shared
//                        memory (or HBM), mixed mechanisms by per-cell id.
//  * rates / jacobian / lu / lusolve kernels — the parity entry points.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>

#include "gf_device.cuh"
#include "gf_internal.h"
#include "gf_persist.cuh"

namespace gf {

// ------------------------------------------------------------ solve kernels

__global__ void __launch_bounds__(128) plain_kernel(const MechSet P, const LaunchArgs a) {
    const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= a.n_cells) return;
    Grp<1> g;
    const DevMech* M = pick(P, a, cell);
    if (!M) {
        reject_cell(g, a, cell);
        return;
    }
    WsS w{a.ws + cell, a.ws_slot_stride};
    process_cell(g, *M, w, a, (int)cell);
}

__global__ void reset_kernel(unsigned long long* q) {
    q[0] = 0;
    q[1] = 0xFFFFFFFFFFFFFFFFull;
    q[2] = 0;
    q[3] = 0;
    q[4] = 0;
}

// ------------------------------------------------------------ parity kernels

__global__ void __launch_bounds__(32) rates_kernel(const DevMech M, const double* y, double* dydx) {
    extern __shared__ double smem[];
    Grp<32> g;
    const WsLayout L = make_layout(M.nS, M.nR, M.n_slots, M.n_tb);
    const int n = M.nS + 2;
    const double* yi = y + (size_t)blockIdx.x * n;
    WsC w{smem};
    for (int i = g.lane; i < M.m; i += 32) w[L.y0 + i] = yi[i];
    const double p = yi[M.nS + 1];
    derivatives(g, M, w, L, L.y0, p, L.dydx);
    double* o = dydx + (size_t)blockIdx.x * n;
    for (int i = g.lane; i < M.m; i += 32) o[i] = w[L.dydx + i];
    if (g.lane == 0) o[n - 1] = 0.0;
}

__global__ void __launch_bounds__(32) jacobian_kernel(const DevMech M, const double* y, double* dfdx, double* J) {
    extern __shared__ double smem[];
    Grp<32> g;
    const WsLayout L = make_layout(M.nS, M.nR, M.n_slots, M.n_tb);
    const int n = M.nS + 2;
    const double* yi = y + (size_t)blockIdx.x * n;
    WsC w{smem};
    for (int i = g.lane; i < M.m; i += 32) w[L.y0 + i] = yi[i];
    const double p = yi[M.nS + 1];
    jacobian(g, M, w, L, L.y0, p);
    double* o = dfdx + (size_t)blockIdx.x * n;
    for (int i = g.lane; i < M.m; i += 32) o[i] = w[L.dfdx + i];
    if (g.lane == 0) o[n - 1] = 0.0;
    double* Jo = J + (size_t)blockIdx.x * n * n;
    for (int e = g.lane; e < n * n; e += 32) {
        const int i = e / n, j = e % n;
        Jo[e] = (i < M.m && j < M.m) ? w[L.J + i * L.ld + j] : 0.0;
    }
}

__global__ void __launch_bounds__(32) lu_kernel(int m, double* A, int* piv) {
    extern __shared__ double smem[];
    Grp<32> g;
    const int ld = m | 1;
    WsC w{smem};
    const int oA = 0, ovv = m * ld, opiv = ovv + m;
    double* Ag = A + (size_t)blockIdx.x * m * m;
    for (int e = g.lane; e < m * m; e += 32) w[oA + (e / m) * ld + (e % m)] = Ag[e];
    g.sync();
    row_scale(g, w, oA, ld, ovv, m);
    lu_decompose(g, w, oA, ld, opiv, ovv, m);
    for (int e = g.lane; e < m * m; e += 32) Ag[e] = w[oA + (e / m) * ld + (e % m)];
    for (int i = g.lane; i < m; i += 32) piv[(size_t)blockIdx.x * m + i] = w.ip(opiv + i);
}

__global__ void __launch_bounds__(32) lusolve_kernel(int m, const double* LU, const int* piv, double* b) {
    extern __shared__ double smem[];
    Grp<32> g;
    const int ld = m | 1;
    WsC w{smem};
    const int oA = 0, ob = m * ld, opiv = ob + m;
    const double* Ag = LU + (size_t)blockIdx.x * m * m;
    for (int e = g.lane; e < m * m; e += 32) w[oA + (e / m) * ld + (e % m)] = Ag[e];
    for (int i = g.lane; i < m; i += 32) {
        w[ob + i] = b[(size_t)blockIdx.x * m + i];
        w.ip(opiv + i) = piv[(size_t)blockIdx.x * m + i];
    }
    lu_solve(g, w, oA, ld, opiv, m, ob);
    for (int i = g.lane; i < m; i += 32) b[(size_t)blockIdx.x * m + i] = w[ob + i];
}

// The factorisation and the solves exactly as the solve kernels run them
// (lu_factor, lu_solve_any) with a group of G threads per matrix: after the
// row scaling of LUDecompose, the register-panel form (G >= 32, m <= 64) or the
// blocked one, reciprocal pivots for G >= 16; EXACT rounds every update a - l u
// twice, as the reference's CPU build does. One matrix per CTA; A [m][m] is
// replaced by its factors, b [n_rhs][m] by the solutions.
template <int G, bool EXACT>
__global__ void __launch_bounds__(G < 32 ? 32 : G) lu_form_kernel(int m, double* A, int* piv, double* b, int n_rhs) {
    extern __shared__ double smem[];
    Grp<G> g;
    if (G < 32 && threadIdx.x >= G) return;
    const int ld = m | 1;
    WsC w{smem};
    const int oA = 0, ovv = m * ld, opiv = ovv + m, operm = opiv + m, ob = operm + m;
    double* Ag = A + (size_t)blockIdx.x * m * m;
    for (int e = g.lane; e < m * m; e += G) w[oA + (e / m) * ld + (e % m)] = Ag[e];
    g.sync();
    row_scale(g, w, oA, ld, ovv, m);
    lu_factor<G, EXACT>(g, w, oA, ld, opiv, ovv, operm, m);
    g.sync();
    for (int e = g.lane; e < m * m; e += G) Ag[e] = w[oA + (e / m) * ld + (e % m)];
    for (int i = g.lane; i < m; i += G) piv[(size_t)blockIdx.x * m + i] = w.ip(opiv + i);
    for (int r = 0; r < n_rhs; ++r) {
        double* bg = b + ((size_t)blockIdx.x * n_rhs + r) * m;
        g.sync();
        for (int i = g.lane; i < m; i += G) w[ob + i] = bg[i];
        g.sync();
        lu_solve_any(g, w, oA, ld, opiv, operm, ovv, m, ob);
        g.sync();
        for (int i = g.lane; i < m; i += G) bg[i] = w[ob + i];
    }
}

template <int G, bool EXACT>
static int launch_lu_form_g(int n_mats, int m, double* A, int* piv, double* b, int n_rhs, cudaStream_t s) {
    const size_t smem = ((size_t)m * (m | 1) + 4 * (size_t)m) * sizeof(double);
    const void* fn = reinterpret_cast<const void*>(&lu_form_kernel<G, EXACT>);
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
    lu_form_kernel<G, EXACT><<<n_mats, G < 32 ? 32 : G, smem, s>>>(m, A, piv, b, n_rhs);
    return (int)cudaGetLastError();
}

template <int G>
static int launch_lu_form_e(int n_mats, int m, double* A, int* piv, double* b, int n_rhs, int exact,
                            cudaStream_t s) {
    return exact ? launch_lu_form_g<G, true>(n_mats, m, A, piv, b, n_rhs, s)
                 : launch_lu_form_g<G, false>(n_mats, m, A, piv, b, n_rhs, s);
}

// ---------------------------------------------------------------- launchers

int launch_lu_form(int n_mats, int m, double* A, int* piv, double* b, int n_rhs, int G, int exact, void* stream) {
    if (n_mats <= 0) return 0;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    switch (G) {
    case 1: return launch_lu_form_e<1>(n_mats, m, A, piv, b, n_rhs, exact, s);
    case 4: return launch_lu_form_e<4>(n_mats, m, A, piv, b, n_rhs, exact, s);
    case 8: return launch_lu_form_e<8>(n_mats, m, A, piv, b, n_rhs, exact, s);
    case 16: return launch_lu_form_e<16>(n_mats, m, A, piv, b, n_rhs, exact, s);
    case 32: return launch_lu_form_e<32>(n_mats, m, A, piv, b, n_rhs, exact, s);
    case 64: return launch_lu_form_e<64>(n_mats, m, A, piv, b, n_rhs, exact, s);
    case 96: return launch_lu_form_e<96>(n_mats, m, A, piv, b, n_rhs, exact, s);
    case 128: return launch_lu_form_e<128>(n_mats, m, A, piv, b, n_rhs, exact, s);
    case 256: return launch_lu_form_e<256>(n_mats, m, A, piv, b, n_rhs, exact, s);
    default: return (int)cudaErrorInvalidValue;
    }
}

WsLayout ws_layout(const DevMech& m) { return make_layout(m.nS, m.nR, m.n_slots, m.n_tb); }

int device_sm_count() {
    int dev = 0, n = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    return n;
}

// The matrix size the tuned kernels are compiled for when every mechanism of a
// launch has it (10-, 53- and 100-species mechanisms), else 0.
int specialized_size(const DevMech* mechs, int n_mechs) {
    if (n_mechs < 1) return 0;
    const int m = mechs[0].m;
    for (int i = 1; i < n_mechs; ++i)
        if (mechs[i].m != m) return 0;
    return (m == 11 || m == 54 || m == 101) ? m : 0;
}

// The persistent kernel of a launch form: the generic variants of every group
// size, or (lu_panel 4 / 16, or specialize with the matrix size ms) the tuned
// variants of the 32-, 64-, 96- and 128-thread forms; nullptr if not compiled.
static const void* persistent_fn(const gf_launch_config& cfg, int ms) {
    const int G = cfg.threads_per_cell;
    const bool shared = cfg.scratch_in_shared != 0;
    const int slim = cfg.register_budget;
    const int nb = (cfg.lu_panel == 0) ? 8 : cfg.lu_panel;
    const int sms = cfg.specialize ? ms : 0;
    if (cfg.specialize && sms == 0) return nullptr;
    if (nb != 8 || sms != 0) {
        switch (G) {
        case 32: return persistent_tuned_fn_g32(shared, slim, nb, sms);
        case 64: return persistent_tuned_fn_g64(shared, slim, nb, sms);
        case 96: return persistent_tuned_fn_g96(shared, slim, nb, sms);
        case 128: return persistent_tuned_fn_g128(shared, slim, nb, sms);
        default: return nullptr;
        }
    }
    switch (G) {
    case 1: return persistent_fn_g1(shared, slim);
    case 2: return persistent_fn_g2(shared, slim);
    case 4: return persistent_fn_g4(shared, slim);
    case 8: return persistent_fn_g8(shared, slim);
    case 16: return persistent_fn_g16(shared, slim);
    case 32: return persistent_fn_g32(shared, slim);
    case 64: return persistent_fn_g64(shared, slim);
    case 96: return persistent_fn_g96(shared, slim);
    case 128: return persistent_fn_g128(shared, slim);
    case 256: return persistent_fn_g256(shared, slim);
    default: return nullptr;
    }
}

bool persistent_form_compiled(const gf_launch_config& cfg, int ms) { return persistent_fn(cfg, ms) != nullptr; }

int persistent_slots(const gf_launch_config& cfg, int ms, int smem_bytes_per_cell, int* blocks_out,
                     int* threads_out) {
    const int G = cfg.threads_per_cell;
    const bool shared = cfg.scratch_in_shared != 0;
    const void* fn = persistent_fn(cfg, ms);
    if (!fn) return -1;
    // G <= 32: several groups per CTA of at most 128 threads; G > 32: one group
    int cpb = G > 32 ? 1 : (cfg.cells_per_block > 0 ? cfg.cells_per_block : std::max(1, 128 / G));
    int threads = cpb * G;
    if (G <= 32 && threads > 128) {
        cpb = 128 / G;
        threads = cpb * G;
    }
    size_t smem = shared ? (size_t)cpb * smem_bytes_per_cell : 0;
    if (smem > 227 * 1024) {
        cpb = std::max(1, (int)((227 * 1024) / smem_bytes_per_cell));
        threads = cpb * G;
        smem = (size_t)cpb * smem_bytes_per_cell;
        if (smem > 227 * 1024) return -2;
    }
    if (shared) cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    // shared-memory carveout: just enough for the CTAs that are resident
    // (blocks_per_sm, or as many as registers, threads and shared memory allow
    // at the largest carveout), so that the rest of the SM's 256 KB serves as
    // L1 for the mechanism tables (with the workspace in HBM: for the
    // workspaces too). The occupancy is taken again at the chosen carveout and
    // the largest one kept if fewer CTAs would fit.
    cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem) != cudaSuccess) return -3;
    if (per_sm <= 0) return -4;
    if (cfg.blocks_per_sm > 0) per_sm = std::min(per_sm, cfg.blocks_per_sm);
    {
        int dev = 0, sm_max = 0, reserved = 0;
        cudaFuncAttributes fa{};
        if (cudaGetDevice(&dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&sm_max, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev) == cudaSuccess &&
            cudaFuncGetAttributes(&fa, fn) == cudaSuccess && sm_max > 0) {
            const size_t need = (size_t)per_sm * (smem + fa.sharedSizeBytes + (size_t)reserved) + (size_t)reserved;
            const int carve = (int)std::min<size_t>(100, (need * 100 + sm_max - 1) / (size_t)sm_max);
            cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, carve);
            int again = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&again, fn, threads, smem) != cudaSuccess ||
                again < per_sm)
                cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        }
    }
    const int blocks = per_sm * device_sm_count();
    *blocks_out = blocks;
    *threads_out = threads;
    return blocks * cpb;
}

int launch_cells(const DevMech* mechs, int n_mechs, const gf_launch_config& cfg, const LaunchArgs& a,
                 int ws_doubles_per_cell, int n_slots_total, void* stream) {
    MechSet P;
    P.n = std::min(n_mechs, kMaxMechs);
    for (int i = 0; i < n_mechs && i < kMaxMechs; ++i) P.m[i] = mechs[i];
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    reset_kernel<<<1, 1, 0, s>>>(a.queue);
    if (a.n_cells <= 0) return (int)cudaGetLastError();
    if (cfg.kind == 0) {
        const int threads = 128;
        const long long blocks = (a.n_cells + threads - 1) / threads;
        plain_kernel<<<(unsigned)blocks, threads, 0, s>>>(P, a);
        return (int)cudaGetLastError();
    }
    const int G = cfg.threads_per_cell;
    const bool shared = cfg.scratch_in_shared != 0;
    int blocks = 0, threads = 0;
    const int ms = specialized_size(mechs, n_mechs);
    const int slots = persistent_slots(cfg, ms, ws_doubles_per_cell * (int)sizeof(double), &blocks, &threads);
    if (slots <= 0) return (int)cudaErrorInvalidConfiguration;
    if (!shared && slots > n_slots_total) return (int)cudaErrorInvalidValue;
    const size_t smem = shared ? (size_t)(threads / G) * ws_doubles_per_cell * sizeof(double) : 0;
    const long long n_slots = slots;
    void* args[] = {(void*)&P, (void*)&a, (void*)&ws_doubles_per_cell, (void*)&n_slots};
    return (int)cudaLaunchKernel(persistent_fn(cfg, ms), dim3(blocks), dim3(threads), args,
                                 smem, s);
}

int launch_rates(const DevMech& m, int n, const double* y, double* dydx, void* stream) {
    if (n <= 0) return 0;
    const size_t smem = (size_t)ws_layout(m).size * sizeof(double);
    cudaFuncSetAttribute(reinterpret_cast<const void*>(&rates_kernel), cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
    rates_kernel<<<n, 32, smem, reinterpret_cast<cudaStream_t>(stream)>>>(m, y, dydx);
    return (int)cudaGetLastError();
}

int launch_jacobian(const DevMech& m, int n, const double* y, double* dfdx, double* J, double* /*ws*/,
                    void* stream) {
    if (n <= 0) return 0;
    const size_t smem = (size_t)ws_layout(m).size * sizeof(double);
    cudaFuncSetAttribute(reinterpret_cast<const void*>(&jacobian_kernel),
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    jacobian_kernel<<<n, 32, smem, reinterpret_cast<cudaStream_t>(stream)>>>(m, y, dfdx, J);
    return (int)cudaGetLastError();
}

int launch_lu(int n_mats, int m, double* A, int* piv, double* /*vv*/, void* stream) {
    if (n_mats <= 0) return 0;
    const size_t smem = ((size_t)m * (m | 1) + 2 * m) * sizeof(double);
    cudaFuncSetAttribute(reinterpret_cast<const void*>(&lu_kernel), cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
    lu_kernel<<<n_mats, 32, smem, reinterpret_cast<cudaStream_t>(stream)>>>(m, A, piv);
    return (int)cudaGetLastError();
}

int launch_lusolve(int n_mats, int m, const double* LU, const int* piv, double* b, void* stream) {
    if (n_mats <= 0) return 0;
    const size_t smem = ((size_t)m * (m | 1) + 2 * m) * sizeof(double);
    cudaFuncSetAttribute(reinterpret_cast<const void*>(&lusolve_kernel),
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    lusolve_kernel<<<n_mats, 32, smem, reinterpret_cast<cudaStream_t>(stream)>>>(m, LU, piv, b);
    return (int)cudaGetLastError();
}

#ifdef GF_PHASE_TIMERS
}  // namespace gf
// Phase-timer cycles summed over every kernel translation unit (profiling
// builds only).
extern "C" int gf_debug_phase_cycles(unsigned long long* out, int reset) {
    using namespace gf;
    for (int i = 0; i < 20; ++i) out[i] = 0;
    phase_cycles_local(out, reset);
    phase_cycles_g1(out, reset);
    phase_cycles_g2(out, reset);
    phase_cycles_g4(out, reset);
    phase_cycles_g8(out, reset);
    phase_cycles_g16(out, reset);
    phase_cycles_g32(out, reset);
    phase_cycles_g64(out, reset);
    phase_cycles_g96(out, reset);
    phase_cycles_g128(out, reset);
    phase_cycles_adj(out, reset);
    phase_cycles_g32t(out, reset);
    phase_cycles_g64t(out, reset);
    phase_cycles_g96t(out, reset);
    phase_cycles_g128t(out, reset);
    return phase_cycles_g256(out, reset);
}
namespace gf {
#endif

int launch_epilogue_reset(unsigned long long* queue, void* stream) {
    reset_kernel<<<1, 1, 0, reinterpret_cast<cudaStream_t>(stream)>>>(queue);
    return (int)cudaGetLastError();
}

}  // namespace gf
