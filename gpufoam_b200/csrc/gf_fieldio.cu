// The plugin's host glue on the device: the gather of OpenFOAM's per-species
// fields into the solve's cell-major states (getY0,
// gpuChemistryModels/gpuChemistryModel/gpuChemistryModel.C:33-53) and the
// scatter of the cell-major rates back into per-species fields
// (computeRRAndChemDeltaT, gpuChemistryModel.C:351-356). Both are transposes
// through a shared-memory tile of kTileCells cells, so that the field-side
// accesses (consecutive cells of one field) and the cell-side accesses
// (consecutive entries of one cell's row) are both coalesced. HBM-bound data
// movement, no arithmetic.
#include <algorithm>

#include "gf_internal.h"

namespace gf {

namespace {

constexpr int kTileCells = 16;
constexpr int kTileThreads = 256;

struct FieldPtrs {
    const double* p[GF_MAX_SPECIES];
};
struct FieldOutPtrs {
    double* p[GF_MAX_SPECIES];
};

// y[c * ld + e] = field_e[c], e < nS the species, nS T, nS + 1 p
__global__ void __launch_bounds__(kTileThreads)
    gather_states_kernel(const FieldPtrs Y, const double* T, const double* p, int n, int nS, double* y, int ld) {
    extern __shared__ double tile[];  // [kTileCells][ne]
    const int ne = nS + 2;
    for (long long c0 = (long long)blockIdx.x * kTileCells; c0 < n; c0 += (long long)gridDim.x * kTileCells) {
        const int nc = n - c0 < kTileCells ? (int)(n - c0) : kTileCells;
        for (int t = threadIdx.x; t < ne * kTileCells; t += blockDim.x) {
            const int e = t / kTileCells, j = t % kTileCells;
            if (j < nc) {
                const double* src = e < nS ? Y.p[e] : (e == nS ? T : p);
                tile[j * ne + e] = src[c0 + j];
            }
        }
        __syncthreads();
        for (int t = threadIdx.x; t < nc * ne; t += blockDim.x) {
            const int j = t / ne, e = t % ne;
            y[(c0 + j) * ld + e] = tile[j * ne + e];
        }
        __syncthreads();
    }
}

// field_i[c] = RR[c * ld + i], i < nS
__global__ void __launch_bounds__(kTileThreads)
    scatter_rates_kernel(const double* RR, int ld, int n, int nS, const FieldOutPtrs out) {
    extern __shared__ double tile[];  // [kTileCells][nS]
    for (long long c0 = (long long)blockIdx.x * kTileCells; c0 < n; c0 += (long long)gridDim.x * kTileCells) {
        const int nc = n - c0 < kTileCells ? (int)(n - c0) : kTileCells;
        for (int t = threadIdx.x; t < nc * nS; t += blockDim.x) {
            const int j = t / nS, i = t % nS;
            tile[j * nS + i] = RR[(c0 + j) * ld + i];
        }
        __syncthreads();
        for (int t = threadIdx.x; t < nS * kTileCells; t += blockDim.x) {
            const int i = t / kTileCells, j = t % kTileCells;
            if (j < nc) out.p[i][c0 + j] = tile[j * nS + i];
        }
        __syncthreads();
    }
}

long long tile_grid(int n) {
    const long long tiles = (n + kTileCells - 1) / kTileCells;
    return std::min<long long>(tiles, 16LL * device_sm_count());
}

}  // namespace

int launch_gather_states(int n, int nS, const double* const* Y, const double* T, const double* p, double* y, int ld,
                         void* stream) {
    if (n <= 0) return 0;
    FieldPtrs P{};
    for (int i = 0; i < nS; ++i) P.p[i] = Y[i];
    const size_t smem = (size_t)kTileCells * (nS + 2) * sizeof(double);
    gather_states_kernel<<<(unsigned)tile_grid(n), kTileThreads, smem, reinterpret_cast<cudaStream_t>(stream)>>>(
        P, T, p, n, nS, y, ld);
    return (int)cudaGetLastError();
}

int launch_scatter_rates(int n, int nS, const double* RR, int ld, double* const* out, void* stream) {
    if (n <= 0) return 0;
    FieldOutPtrs P{};
    for (int i = 0; i < nS; ++i) P.p[i] = out[i];
    const size_t smem = (size_t)kTileCells * nS * sizeof(double);
    scatter_rates_kernel<<<(unsigned)tile_grid(n), kTileThreads, smem, reinterpret_cast<cudaStream_t>(stream)>>>(
        RR, ld, n, nS, P);
    return (int)cudaGetLastError();
}

}  // namespace gf
