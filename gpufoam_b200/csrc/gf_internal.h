// Internal declarations shared by the host code (gf_host.cpp) and the CUDA
// kernels (gf_kernels.cu). Not part of the public C ABI.
#pragma once

#include <cstdint>
#include <vector>

#include "../../include/gpufoam_b200.h"

namespace gf {

constexpr int kMaxW = GF_MAX_REACTION_WIDTH;
constexpr int kNoIntExp = 2147483647 / 10;  // gpuLabelMax: "not an integer exponent"

// Packed per-reaction data (compute order q), loaded with a handful of
// independent 16-byte loads: the head and up to kSideInline species per side.
struct __align__(16) RxnHead {
    int type, irr, slot, tb_row;   // tb_row: row of eff, -1 for plain Arrhenius
    int nl, nr, sp_off, nm_small;  // nm_small: Kc = K (gpuThermo.H:111)
    double lnA0, beta0, Ta0, sA0;  // k (or the fall-off k0): ln|A|, beta, Ta, sign(A)
    double Tcommon, Y, nm, pad;    // the reaction ΔThermo's Tcommon, Y and Y / W
};
constexpr int kSideInline = 4;
// species entry of a reaction side: index, integer exponent (or kNoIntExp), exponent
struct __align__(16) RxnSpecie {
    int idx;
    int iexp;
    double exp;
};

// One record of a gather stream: acc += coef * src[slot] (slot < 0: nothing);
// pos >= 0 marks the last record of an output entry: dst[pos] = acc, acc = 0.
struct __align__(16) StreamRec {
    int pos;
    int slot;
    double coef;
};

// The records of a gather y[pos] = sum coef * x[slot], entry by entry in the
// reference's summation order, split over G threads (entries balanced by
// record count) and interleaved: record k of thread t is rec[k * G + t], so
// a warp's loads are coalesced and every load is independent of the sums.
struct Stream {
    const StreamRec* rec;
    int len;  // records per thread (padded)
};
constexpr int kNumGroupSizes = 10;  // G = 1, 2, 4, ..., 256: stream index log2(G); G = 96: index 9
constexpr int group_size_of(int k) { return k < 9 ? 1 << k : 96; }

// Device-resident mechanism tables. All arrays are device pointers; the struct
// itself is passed to kernels by value.
//
// Layout (nS species, nR reactions, m = nS + 1 unknowns of the linear
// algebra: the pressure row and column of the reference Jacobian are
// identically zero, gpuODESystem.H:101 and :195, so the solve runs on Y and T):
//  * species NASA-7 coefficients: coef[(b * 7 + k) * nS + i], b = 0 low / 1 high
//  * reactions are stored in "compute order" q (grouped by rate type, so that
//    the lanes of a warp evaluate reactions of one kind together and read
//    consecutive table entries); rcoef[(b * 7 + k) * nR + q] is the reaction
//    ΔThermo. Arrhenius factors are kept as ln|A| and sign(A) (log-space
//    evaluation k = sign * exp(ln|A| + beta ln T - Ta / T)); index 0 is k (or the
//    fall-off k0), index 1 the fall-off kInf.
//  * stoichiometry: compact CSR, sp_off[q] .. + nl[q] (lhs) + nr[q] (rhs)
//  * staging slots of reaction q start at slot[q]:
//      [0] omega, [1] dwdT, [2 .. 2+nl) dCf*kf, [2+nl .. 2+nl+nr) dCr*kr,
//      third body only: [2+nl+nr] Ak * (Cf - Cr/Kc)
//  * dst[log2 G]: the gather streams of dN_s/dt: per species s the (omega slot,
//    signed stoich) terms in mechanism order (gpuReaction.H:490-508)
//  * jst[log2 G]: the gather streams of the raw Jacobian: entry (row s,
//    column c < nS or the T column c = nS), position s * ld + c in the
//    workspace Jacobian, takes its dN/dc, T-column and third-body terms in the
//    reference's update order (gpuReaction.H:547-648 over reactions in
//    mechanism order). A third-body term is (stoich * eff_c) * (Ak * (Cf -
//    Cr/Kc)) (the reference: stoich * ((eff_c * Ak) * (Cf - Cr/Kc))).
struct DevMech {
    int nS, nR, m;
    int n_slots;
    int n_tb;
    double Tlow, Thigh;        // reaction temperature limits (uniform)
    // species
    const double* W;
    const double* Rsp;         // RR / W
    const double* Tcommon;
    const double* coef;
    const double* hf;          // enthalpy of formation [J/kg] (Qdot)
    // reactions, compute order
    const int* rtype;
    const int* rirr;
    const int* nl;
    const int* nr;
    const int* sp_off;
    const int* slot;
    const double* rY;          // ΔThermo Y
    const double* rnm;         // Y / W
    const int* rnm_small;      // Kc = K when nm is "small" (gpuThermo.H:111)
    const double* rTcommon;
    const double* rcoef;
    const double* lnA0;
    const double* sA0;
    const double* beta0;
    const double* Ta0;
    const double* lnA1;
    const double* sA1;
    const double* beta1;
    const double* Ta1;
    const double* troe;        // [nR][4]: alpha, 1/Tsss, 1/Ts, Tss
    const int* tb_row;         // [nR] row of eff, -1 for plain Arrhenius
    const double* eff;         // [n_tb][nS]
    const int* r_of_q;         // [nR] mechanism index of the reaction in compute position q
    const RxnHead* rxh;        // [nR]
    const RxnSpecie* rxs;      // [nR][2 * kSideInline]: lhs, then rhs (wider sides: sidx/siexp/sexp)
    const int* sidx;
    const int* siexp;          // integer exponent or kNoIntExp
    const double* sst;
    const double* sexp;
    Stream dst[kNumGroupSizes];
    Stream jst[kNumGroupSizes];
    // the adjoint's concentration gathers: per species s, the per-reaction
    // entry slots q * 2 * kSideInline + e whose species is s
    Stream cst[kNumGroupSizes];
    int max_side;              // most species on one side of a reaction
};

struct OdeParams {
    int solver;
    double absTol, relTol;
    int maxSteps;
    double safeScale, alphaInc, alphaDec, minScale, maxScale;
};

// Per-cell workspace layout (in doubles) for a mechanism.
struct WsLayout {
    int ld;          // Jacobian / LU row stride (odd, bank-conflict free columns)
    int J, y0, yt, dydx0, dydx, dfdx, k1, k2, k3, k4, c, Cp, Ha, rhoMbyW, vj, vv, piv, perm, stage, Mtb, scal;
    int size;        // total doubles
};

WsLayout ws_layout(const DevMech& m);

struct LaunchArgs {
    int n_cells;
    double deltaT;
    const double* deltaT_cell;
    double deltaTChemMax;
    const int* mech_id;
    const double* rho;
    const double* Y0;
    int ld_y;
    double* Ynew;
    double* deltaTChem;
    double* RR;
    int ld_rr;
    int* status;
    int* counters;
    double Treact;
    OdeParams ode;
    // device-side scratch owned by the solver
    double* ws;                    // workspaces
    long long ws_slot_stride;      // doubles per slot (blocked) or number of slots (interleaved)
    unsigned long long* queue;     // [0] next cell, [1] min deltaTChem bits, [2] accepted, [3] attempts, [4] failed
    // optional trajectory record (the adjoint's forward pass): for accepted
    // step k of a cell, traj[(cell * traj_cap + k) * traj_ld + 0 .. m) = the
    // state at its start and [m] = its step size; a cell that takes more than
    // traj_cap accepted steps records the first traj_cap and reports MAX_STEPS
    double* traj = nullptr;
    int traj_cap = 0;
    int traj_ld = 0;
};

// Kernel launchers (gf_kernels.cu). All return a cudaError_t as int.
int launch_cells(const DevMech* mechs, int n_mechs, const gf_launch_config& cfg, const LaunchArgs& a,
                 int ws_doubles_per_cell, int n_slots_total, void* stream);
int launch_rates(const DevMech& m, int n, const double* y, double* dydx, void* stream);
int launch_jacobian(const DevMech& m, int n, const double* y, double* dfdx, double* J, double* ws,
                    void* stream);
int launch_lu(int n_mats, int m, double* A, int* piv, double* vv, void* stream);
int launch_lusolve(int n_mats, int m, const double* LU, const int* piv, double* b, void* stream);
// The production factorisation and solves (lu_factor, lu_solve_any) with G threads per matrix.
int launch_lu_form(int n_mats, int m, double* A, int* piv, double* b, int n_rhs, int G, int exact, void* stream);
int launch_epilogue_reset(unsigned long long* queue, void* stream);

// The discrete adjoint (gf_adjoint.cu).
struct AdjArgs;
int adjoint_ws_doubles(const DevMech& m);
int launch_adjoint_cells(const DevMech& m, int n_cells, const double* traj, int traj_cap, const int* counters,
                         const int* fwd_status, const double* Y0, const double* Ynew, const double* Ybar, int ld_y,
                         double* Y0bar, double* theta_bar, int* status, const OdeParams& ode, double* ws,
                         long long ws_per_cell, int n_blocks, unsigned long long* queue, void* stream);
int adjoint_blocks_per_sm(const DevMech& m);
int launch_record(const DevMech& m, const LaunchArgs& a, void* stream);

// The plugin's per-cell side paths (gf_fields.cu).
struct FieldArgs {
    int n_cells;
    const double* rho;
    const double* y;
    int ld_y;
    double* RR;        // calculate() / specieReactionRR(r) [n][ld_rr] or null
    int ld_rr;
    double* tc;        // tc() [n] or null
    int reaction;      // >= 0: reactionRR / specieReactionRR of this reaction
    int reaction_q;    // its compute position
    double* omega;     // reactionRR(r) [n] or null
};
int launch_cell_fields(const DevMech& m, const FieldArgs& a, void* stream);
int launch_qdot(const DevMech& m, int n_cells, const double* RR, int ld_rr, double* qdot, void* stream);

// The plugin's field gather and rate scatter (gf_fieldio.cu).
int launch_gather_states(int n, int nS, const double* const* Y, const double* T, const double* p, double* y, int ld,
                         void* stream);
int launch_scatter_rates(int n, int nS, const double* RR, int ld, double* const* out, void* stream);

// Device tables of a mechanism object and the device that holds them (gf_host.cpp).
const DevMech* mech_device_tables(const gf_mech* m);
int mech_device(const gf_mech* m);
// Keeps the CUDA error's text for gf_last_cuda_error and returns its gf_status.
int record_cuda_error(int cuda_error);

// Resident-slot count for a persistent configuration (groups that run at once).
// ms: specialized_size of the launch's mechanisms.
int persistent_slots(const gf_launch_config& cfg, int ms, int smem_bytes_per_cell, int* blocks_out,
                     int* threads_out);
int specialized_size(const DevMech* mechs, int n_mechs);
// Whether the library compiles the persistent kernel of this launch form.
bool persistent_form_compiled(const gf_launch_config& cfg, int ms);
int device_sm_count();

}  // namespace gf
