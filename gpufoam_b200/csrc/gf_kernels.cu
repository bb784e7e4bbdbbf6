// Kernels and launchers of the per-cell chemistry path (sm_100a).
//
//  * plain_kernel      — one thread per cell, one launch over all cells, per-cell
//                        scratch interleaved in HBM: the reference's launch model
//                        (for_each_index.H:25-48, singleCellSolver.H:27-51) with
//                        coalesced scratch.
//  * persistent_kernel — one CTA set sized to the SMs; groups of G threads pull
//                        cells from an atomic work queue, scratch in shared memory
//                        (or HBM), mixed mechanisms by per-cell id.
//  * rates / jacobian / lu / lusolve kernels — the parity entry points.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>

#include "gf_device.cuh"
#include "gf_internal.h"

namespace gf {

constexpr int kMaxMechs = 4;

struct MechSet {
    DevMech m[kMaxMechs];
    int n;
};

__device__ __forceinline__ const DevMech& pick(const MechSet& P, const LaunchArgs& a, long long cell) {
    const int id = a.mech_id ? a.mech_id[cell] : 0;
    return P.m[id];
}

// ------------------------------------------------------------ solve kernels

__global__ void __launch_bounds__(128) plain_kernel(const MechSet P, const LaunchArgs a) {
    const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= a.n_cells) return;
    Grp<1> g;
    const DevMech& M = pick(P, a, cell);
    WsS w{a.ws + cell, a.ws_slot_stride};
    process_cell(g, M, w, a, (int)cell);
}

// MINB = 1: up to 255 registers per thread (fewer resident groups, no spills);
// MINB = 4: at most 128 registers (more resident groups).
template <int G, bool SHARED, int MINB>
__global__ void __launch_bounds__(128, MINB) persistent_kernel(const MechSet P, const LaunchArgs a, int ws_per_cell,
                                                               long long n_slots) {
    extern __shared__ double smem[];
    Grp<G> g;
    const int gpb = blockDim.x / G;
    const int gib = threadIdx.x / G;
    const long long slot = (long long)blockIdx.x * gpb + gib;
    for (;;) {
        long long cell = 0;
        if (g.lane == 0) cell = (long long)atomicAdd(a.queue, 1ull);
        cell = g.bcast_ll(cell, 0);
        if (cell >= a.n_cells) break;
        const DevMech& M = pick(P, a, cell);
        if (SHARED) {
            process_cell(g, M, WsC{smem + (size_t)gib * ws_per_cell}, a, (int)cell);
        } else if (G == 1) {
            process_cell(g, M, WsS{a.ws + slot, n_slots}, a, (int)cell);
        } else {
            process_cell(g, M, WsC{a.ws + slot * ws_per_cell}, a, (int)cell);
        }
    }
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
    const WsLayout L = make_layout(M.nS, M.nR, M.n_slots);
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
    const WsLayout L = make_layout(M.nS, M.nR, M.n_slots);
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

// ---------------------------------------------------------------- launchers

WsLayout ws_layout(const DevMech& m) { return make_layout(m.nS, m.nR, m.n_slots); }

int device_sm_count() {
    int dev = 0, n = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    return n;
}

template <int G, bool SHARED>
static const void* persistent_ptr(int slim) {
    return slim ? reinterpret_cast<const void*>(&persistent_kernel<G, SHARED, 4>)
                : reinterpret_cast<const void*>(&persistent_kernel<G, SHARED, 1>);
}

static const void* persistent_fn(int G, bool shared, int slim) {
    switch (G) {
    case 1: return shared ? persistent_ptr<1, true>(slim) : persistent_ptr<1, false>(slim);
    case 2: return shared ? persistent_ptr<2, true>(slim) : persistent_ptr<2, false>(slim);
    case 4: return shared ? persistent_ptr<4, true>(slim) : persistent_ptr<4, false>(slim);
    case 8: return shared ? persistent_ptr<8, true>(slim) : persistent_ptr<8, false>(slim);
    case 16: return shared ? persistent_ptr<16, true>(slim) : persistent_ptr<16, false>(slim);
    case 32: return shared ? persistent_ptr<32, true>(slim) : persistent_ptr<32, false>(slim);
    default: return nullptr;
    }
}

int persistent_slots(const gf_launch_config& cfg, int smem_bytes_per_cell, int* blocks_out, int* threads_out) {
    const int G = cfg.threads_per_cell;
    const bool shared = cfg.scratch_in_shared != 0;
    const void* fn = persistent_fn(G, shared, cfg.register_budget);
    if (!fn) return -1;
    int cpb = cfg.cells_per_block > 0 ? cfg.cells_per_block : std::max(1, 128 / G);
    int threads = cpb * G;
    if (threads > 128) {
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
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem) != cudaSuccess) return -3;
    if (per_sm <= 0) return -4;
    if (cfg.blocks_per_sm > 0) per_sm = std::min(per_sm, cfg.blocks_per_sm);
    const int blocks = per_sm * device_sm_count();
    *blocks_out = blocks;
    *threads_out = threads;
    return blocks * cpb;
}

int launch_cells(const DevMech* mechs, int n_mechs, const gf_launch_config& cfg, const LaunchArgs& a,
                 int ws_doubles_per_cell, int n_slots_total, void* stream) {
    MechSet P;
    P.n = n_mechs;
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
    const int slots = persistent_slots(cfg, ws_doubles_per_cell * (int)sizeof(double), &blocks, &threads);
    if (slots <= 0) return (int)cudaErrorInvalidConfiguration;
    if (!shared && slots > n_slots_total) return (int)cudaErrorInvalidValue;
    const size_t smem = shared ? (size_t)(threads / G) * ws_doubles_per_cell * sizeof(double) : 0;
    const long long n_slots = slots;
    void* args[] = {(void*)&P, (void*)&a, (void*)&ws_doubles_per_cell, (void*)&n_slots};
    return (int)cudaLaunchKernel(persistent_fn(G, shared, cfg.register_budget), dim3(blocks), dim3(threads), args,
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
extern "C" int gf_debug_phase_cycles(unsigned long long* out, int reset) {
    using gf::g_phase_cycles;
    cudaMemcpyFromSymbol(out, g_phase_cycles, sizeof(unsigned long long) * 16);
    if (reset) {
        unsigned long long z[16] = {};
        cudaMemcpyToSymbol(g_phase_cycles, z, sizeof(z));
    }
    return (int)cudaGetLastError();
}
namespace gf {
#endif

int launch_epilogue_reset(unsigned long long* queue, void* stream) {
    reset_kernel<<<1, 1, 0, reinterpret_cast<cudaStream_t>(stream)>>>(queue);
    return (int)cudaGetLastError();
}

}  // namespace gf
