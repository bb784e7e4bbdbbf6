// gf_solve_noalloc: the per-flow-step chemistry solve without any device
// allocation, for callers that cannot call cudaMalloc: a host code whose device
// memory belongs to another allocator (a caching pool that has reserved the
// free memory, or a host application that requires every allocation to go
// through its own memory manager), or a real-time loop that forbids
// allocation once it has started.
//
// Every other solve entry point keeps its scratch (per-cell workspaces and the
// work-queue counters) in device memory that gf_solver_create / gf_solve
// allocate. Here that scratch is a file-scope static __device__ array of a
// fixed size (kScratchDoubles doubles = 32 MiB, plus 64 bytes of counters): it
// exists on every GPU that loads the library, from module load until process
// exit. The kernel is the persistent work-queue form with one warp per cell;
// the number of resident cell groups is capped so that all their workspaces
// fit in the array.
//
// Host code never passes the arrays' names to a kernel (in host code they are
// host-side stand-ins, not device addresses). The first call on each device
// resolves their device addresses with cudaGetSymbolAddress, with that device
// current, and keeps them for later calls; that first call should therefore
// happen before any stream capture begins.
//
// All calls share the same arrays: the counters are cleared at the start of
// every call (on the caller's stream), the workspaces need no clearing, and
// calls whose kernels overlap on a GPU (different streams, or different host
// threads on the same device) race on the arrays and must not be issued.
//
// With stats != NULL the call copies the step totals to the host and waits for
// the caller's stream; it then refuses a stream that is being captured
// (GF_ERR_INVALID_ARGUMENT), whose capture that wait would invalidate.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "gf_device.cuh"
#include "gf_internal.h"

namespace {

constexpr long long kScratchDoubles = GF_NOALLOC_SCRATCH_BYTES / 8;  // 32 MiB of workspaces
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_ws[kScratchDoubles];
static __device__ __align__(256) unsigned long long g_noalloc_queue[8];

struct SymbolAddrs {
    double* ws = nullptr;
    unsigned long long* queue = nullptr;
};
SymbolAddrs g_addrs[kMaxDevices];
std::mutex g_addrs_mutex;

// One warp per cell, workspace in the static array, at most 128 registers per
// thread (16 one-warp CTAs per SM).
__global__ void __launch_bounds__(32, 16) noalloc_kernel(const gf::DevMech M, const gf::LaunchArgs a,
                                                          int ws_per_cell) {
    gf::Grp<32> g;
    const long long slot = blockIdx.x;
    for (;;) {
        long long cell = 0;
        if (g.lane == 0) cell = (long long)atomicAdd(a.queue, 1ull);
        cell = g.bcast_ll(cell, 0);
        if (cell >= a.n_cells) break;
        gf::process_cell(g, M, gf::WsC{a.ws + slot * ws_per_cell}, a, (int)cell);
    }
}

__global__ void noalloc_reset(unsigned long long* q) {
    q[0] = 0;
    q[1] = 0xFFFFFFFFFFFFFFFFull;
    q[2] = 0;
    q[3] = 0;
    q[4] = 0;
}

int symbol_addresses(int dev, SymbolAddrs* out) {
    if (dev < 0 || dev >= kMaxDevices) return GF_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_addrs_mutex);
    SymbolAddrs& s = g_addrs[dev];
    if (!s.ws) {
        void* ws = nullptr;
        void* q = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ws, g_noalloc_ws);
        if (e == cudaSuccess) e = cudaGetSymbolAddress(&q, g_noalloc_queue);
        if (e != cudaSuccess) return gf::record_cuda_error((int)e);
        s.ws = static_cast<double*>(ws);
        s.queue = static_cast<unsigned long long*>(q);
    }
    *out = s;
    return GF_OK;
}

}  // namespace

extern "C" int gf_solve_noalloc(const gf_mech* mech, const gf_ode_inputs* in, double Treact, int n_cells,
                                double deltaT, const double* deltaT_cell, double deltaTChemMax, const double* rho,
                                const double* Y0, int ld_y, double* Ynew, double* deltaTChem, double* RR, int ld_rr,
                                int* status, int* counters, gf_stats* stats, void* stream) {
    if (!mech || !in || n_cells < 0 || !Y0 || !deltaTChem) return GF_ERR_INVALID_ARGUMENT;
    if (in->solver != GF_ROSENBROCK12 && in->solver != GF_ROSENBROCK23 && in->solver != GF_ROSENBROCK34)
        return GF_ERR_UNKNOWN_SOLVER;
    const gf::DevMech* M = gf::mech_device_tables(mech);
    if (ld_y < M->nS + 2 || (RR && (!rho || ld_rr < M->nS))) return GF_ERR_INVALID_ARGUMENT;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return gf::record_cuda_error((int)e);
    // the mechanism's tables must be on the current device
    if (dev != gf::mech_device(mech)) return GF_ERR_INVALID_ARGUMENT;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (stats) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        e = cudaStreamIsCapturing(s, &cs);
        if (e != cudaSuccess) return gf::record_cuda_error((int)e);
        if (cs != cudaStreamCaptureStatusNone) return GF_ERR_INVALID_ARGUMENT;
    }
    const long long wsd = gf::ws_layout(*M).size;
    // the cap: workspaces of the resident cell groups must fit in the array
    long long groups_fit = kScratchDoubles / wsd;
    if (groups_fit < 1) return GF_ERR_UNSUPPORTED;
    SymbolAddrs addr;
    int r = symbol_addresses(dev, &addr);
    if (r) return r;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, noalloc_kernel, 32, 0);
    if (e != cudaSuccess) return gf::record_cuda_error((int)e);
    if (per_sm < 1) return GF_ERR_UNSUPPORTED;
    const long long groups = std::min<long long>(groups_fit, (long long)per_sm * gf::device_sm_count());
    gf::LaunchArgs a;
    a.n_cells = n_cells;
    a.deltaT = deltaT;
    a.deltaT_cell = deltaT_cell;
    a.deltaTChemMax = deltaTChemMax;
    a.mech_id = nullptr;
    a.rho = rho;
    a.Y0 = Y0;
    a.ld_y = ld_y;
    a.Ynew = Ynew;
    a.deltaTChem = deltaTChem;
    a.RR = RR;
    a.ld_rr = ld_rr;
    a.status = status;
    a.counters = counters;
    a.Treact = Treact;
    a.ode = gf::OdeParams{in->solver, in->absTol, in->relTol, in->maxSteps, in->safeScale, in->alphaInc,
                          in->alphaDec, in->minScale, in->maxScale};
    a.ws = addr.ws;
    a.ws_slot_stride = wsd;
    a.queue = addr.queue;
    noalloc_reset<<<1, 1, 0, s>>>(addr.queue);
    if (n_cells > 0) noalloc_kernel<<<(unsigned)groups, 32, 0, s>>>(*M, a, (int)wsd);
    e = cudaGetLastError();
    if (e != cudaSuccess) return gf::record_cuda_error((int)e);
    if (stats) {
        unsigned long long q[5];
        e = cudaMemcpyAsync(q, addr.queue, sizeof(q), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return gf::record_cuda_error((int)e);
        const unsigned long long k = q[1];
        const unsigned long long bits = (k >> 63) ? (k & 0x7FFFFFFFFFFFFFFFull) : ~k;
        double mn;
        std::memcpy(&mn, &bits, 8);
        stats->min_delta_t = n_cells > 0 ? mn : 0.0;
        stats->accepted_steps = (long long)q[2];
        stats->attempts = (long long)q[3];
        stats->failed_cells = (long long)q[4];
    }
    return GF_OK;
}
