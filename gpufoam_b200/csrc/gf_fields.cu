// The plugin's per-cell side paths on the GPU. The reference computes them on
// the CPU, one cell at a time through OpenFOAM's reactions
// (gpuChemistryModels/gpuChemistryModel/gpuChemistryModel.C):
//   calculate()            :145-186  RR_i = W_i dN_i/dt / V
//   reactionRR(r)          :188-229  omega of reaction r
//   specieReactionRR(r)    :231-298  W_i dN_i/dt / V of reaction r alone
//   tc()                   :366-427  chemical time scale
//   Qdot()                 :429-450  -sum_i hf_i RR_i
// all at the concentrations c_i = rho Y_i / W_i of the thermo's density field
// (:163-166), the rates as gpuReaction::omega computes them
// (gpuReaction.H:472-488: kf Cf - kr Cr at the clipped temperature).
//
// One warp per cell with the cell's concentrations, third-body sums and
// per-reaction staging in shared memory: the same device functions as the
// solve (third_body_all, rate_k, reaction_lnKc, side_C, the dN/dt gather
// stream). Qdot is one thread per cell with the reference's sequential sum.
#include <algorithm>
#include <cfloat>

#include "gf_device.cuh"

namespace gf {

namespace {

constexpr int kFieldCellsMax = 4;  // cells (warps) per CTA

struct FieldLayout {
    WsLayout L;  // only c, Mtb and stage are used
    int out;     // dN/dt of every species
    int size;
};

__host__ __device__ inline FieldLayout field_layout(const DevMech& M) {
    FieldLayout F{};
    int o = 0;
    F.L.c = o;
    o += M.nS;
    F.L.Mtb = o;
    o += M.n_tb > 0 ? M.n_tb : 1;
    F.L.stage = o;
    o += M.n_slots > 0 ? M.n_slots : 1;
    F.out = o;
    o += M.nS;
    F.size = o;
    return F;
}

// Per reaction (compute order, lanes): omega = kf Cf - kr Cr into staging
// slot 0 for the dN/dt gather; with want_tc the lane's shares of tc()'s two
// sums over reactions, sumW and sum of squares (wf = sum_rhs stoich * kf Cf,
// wr = sum_lhs stoich * kr Cr, each counted once in both).
template <class W>
__device__ __forceinline__ void stage_fields(const Grp<32>& g, const DevMech& M, const W& w, const WsLayout& L,
                                             const TCache& tc, bool want_tc, double* sumW, double* sumW2) {
    double sW = 0.0, sW2 = 0.0;
    for (int q = g.lane; q < M.nR; q += 32) {
        Rxn R;
        load_rxn(M, q, R);
        const double Mc = R.tb_row >= 0 ? w[L.Mtb + R.tb_row] : 0.0;
        double dummy, Ak = 0.0;
        const double kf = rate_k(M, q, R, tc, Mc, false, &dummy, &Ak);
        double kr = 0.0;
        if (!R.irr) kr = kf * exp(-reaction_lnKc(M, q, R, tc, nullptr, nullptr));
        const double omegaf = kf * side_C(M, w, L.c, R, 0);
        const double omegar = kr * side_C(M, w, L.c, R, 1);
        w[L.stage + R.slot] = omegaf - omegar;
        if (want_tc) {
            double wf = 0.0, wr = 0.0;
            for (int e = 0; e < R.nr; ++e) wf += ldg(M.sst + R.sp_off + R.nl + e) * omegaf;
            for (int e = 0; e < R.nl; ++e) wr += ldg(M.sst + R.sp_off + e) * omegar;
            sW += wf + wr;
            sW2 += wf * wf + wr * wr;
        }
    }
    *sumW = sW;
    *sumW2 = sW2;
}

__global__ void __launch_bounds__(32 * kFieldCellsMax) cell_fields_kernel(const DevMech M, const FieldArgs a) {
    extern __shared__ double smem[];
    Grp<32> g;
    const FieldLayout F = field_layout(M);
    const int per_cta = blockDim.x >> 5;
    const int warp = threadIdx.x >> 5;
    WsC w{smem + (size_t)warp * F.size};
    const int nS = M.nS;
    for (long long cell = (long long)blockIdx.x * per_cta + warp; cell < a.n_cells;
         cell += (long long)gridDim.x * per_cta) {
        const double* y = a.y + cell * a.ld_y;
        const double rho = a.rho[cell];
        double csum = 0.0;
        for (int i = g.lane; i < nS; i += 32) {
            const double ci = rho * y[i] / ldg(M.W + i);
            w[F.L.c + i] = ci;
            csum += ci;
        }
        g.sync();
        if (M.n_tb > 0) {
            third_body_all(g, M, w, F.L.c, F.L.Mtb);
            g.sync();
        }
        const double T = y[nS];
        const TCache tcache = make_tcache(fmin(fmax(T, M.Tlow), M.Thigh));
        if (a.reaction >= 0) {
            // reactionRR / specieReactionRR: one reaction, lane 0
            double* rr = a.RR ? a.RR + cell * a.ld_rr : nullptr;
            if (rr)
                for (int i = g.lane; i < nS; i += 32) w[F.out + i] = 0.0;
            g.sync();
            if (g.lane == 0) {
                const int q = a.reaction_q;
                Rxn R;
                load_rxn(M, q, R);
                const double Mc = R.tb_row >= 0 ? w[F.L.Mtb + R.tb_row] : 0.0;
                double dummy, Ak = 0.0;
                const double kf = rate_k(M, q, R, tcache, Mc, false, &dummy, &Ak);
                double kr = 0.0;
                if (!R.irr) kr = kf * exp(-reaction_lnKc(M, q, R, tcache, nullptr, nullptr));
                const double om = kf * side_C(M, w, F.L.c, R, 0) - kr * side_C(M, w, F.L.c, R, 1);
                if (a.omega) a.omega[cell] = om;
                if (rr) {
                    // gpuReaction::dNdtByV (gpuReaction.H:490-508): lhs, then rhs
                    for (int e = 0; e < R.nl; ++e) {
                        const int b = R.sp_off + e;
                        w[F.out + ldg(M.sidx + b)] -= ldg(M.sst + b) * om;
                    }
                    for (int e = 0; e < R.nr; ++e) {
                        const int b = R.sp_off + R.nl + e;
                        w[F.out + ldg(M.sidx + b)] += ldg(M.sst + b) * om;
                    }
                }
            }
            g.sync();
            if (rr)
                for (int i = g.lane; i < nS; i += 32) rr[i] = w[F.out + i] * ldg(M.W + i);
            g.sync();
            continue;
        }
        double sW, sW2;
        stage_fields(g, M, w, F.L, tcache, a.tc != nullptr, &sW, &sW2);
        g.sync();
        if (a.RR) {
            stream_gather(g, M.dst[stream_index(32)], w, F.L.stage, F.out);
            g.sync();
            double* rr = a.RR + cell * a.ld_rr;
            for (int i = g.lane; i < nS; i += 32) rr[i] = w[F.out + i] * ldg(M.W + i);
        }
        if (a.tc) {
            const double sumW = g.sum(sW), sumW2 = g.sum(sW2), ctot = g.sum(csum);
            if (g.lane == 0) a.tc[cell] = sumW2 == 0.0 ? DBL_MAX / 10.0 : sumW / sumW2 * ctot;
        }
        g.sync();
    }
}

// Qdot = 0 - hf_0 RR_0 - hf_1 RR_1 - ... in species order, each product
// rounded before the subtraction (no contraction), as the reference's loop.
__global__ void qdot_kernel(const DevMech M, int n, const double* RR, int ld_rr, double* qdot) {
    for (long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x; cell < n;
         cell += (long long)gridDim.x * blockDim.x) {
        const double* r = RR + cell * ld_rr;
        double q = 0.0;
        for (int i = 0; i < M.nS; ++i) q = __dsub_rn(q, __dmul_rn(ldg(M.hf + i), r[i]));
        qdot[cell] = q;
    }
}

}  // namespace

int launch_cell_fields(const DevMech& M, const FieldArgs& a, void* stream) {
    if (a.n_cells <= 0) return 0;
    const FieldLayout F = field_layout(M);
    const size_t per_cell = (size_t)F.size * sizeof(double);
    int dev = 0, max_smem = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    int cells = kFieldCellsMax;
    while (cells > 1 && per_cell * cells > (size_t)max_smem) --cells;
    if (per_cell * cells > (size_t)max_smem) return (int)cudaErrorInvalidValue;
    const size_t smem = per_cell * cells;
    cudaError_t e = cudaFuncSetAttribute(reinterpret_cast<const void*>(&cell_fields_kernel),
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cell_fields_kernel, 32 * cells, smem);
    if (e != cudaSuccess) return (int)e;
    const long long want = (a.n_cells + cells - 1) / cells;
    const long long grid = std::min<long long>(want, (long long)std::max(per_sm, 1) * device_sm_count());
    cell_fields_kernel<<<(unsigned)grid, 32 * cells, smem, reinterpret_cast<cudaStream_t>(stream)>>>(M, a);
    return (int)cudaGetLastError();
}

int launch_qdot(const DevMech& M, int n, const double* RR, int ld_rr, double* qdot, void* stream) {
    if (n <= 0) return 0;
    const int threads = 128;
    const long long grid = std::min<long long>((n + threads - 1) / threads, 8LL * device_sm_count());
    qdot_kernel<<<(unsigned)grid, threads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(M, n, RR, ld_rr, qdot);
    return (int)cudaGetLastError();
}

}  // namespace gf
