// Host side of the C ABI (include/gpufoam_b200.h): mechanism loader arithmetic,
// device mechanism tables, solver objects and the per-flow-step solve.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <new>
#include <string>
#include <vector>

#include "gf_internal.h"

namespace {

// gpu_utils/common/gpu_constants.H:13-82
constexpr double kRR = 6.02214e+26 * 1.38065e-23;
constexpr double kTstd = 298.15;  // gpu_constants.H
constexpr double kSmall = DBL_EPSILON;
constexpr double kVSmall = DBL_MIN;
constexpr double kGreat = 1.0 / DBL_EPSILON;

thread_local std::string g_last_cuda_error;

int cuda_fail(cudaError_t e) {
    g_last_cuda_error = cudaGetErrorString(e);
    if (e == cudaErrorMemoryAllocation) return GF_ERR_OUT_OF_MEMORY;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return GF_ERR_NO_DEVICE;
    return GF_ERR_CUDA;
}

#define GF_CUDA(x)                                  \
    do {                                            \
        cudaError_t e_ = (x);                       \
        if (e_ != cudaSuccess) return cuda_fail(e_); \
    } while (0)

// ---- reference loader arithmetic on gf_thermo (gpuThermo.H:352-470,
//      gpuPerfectGas.H:100-117, 280-325)

void thermo_add(gf_thermo& a, const gf_thermo& b) {
    double Y1 = a.Y;
    const double sumY = a.Y + b.Y;
    if (std::fabs(sumY) > kSmall) a.W = sumY / (a.Y / a.W + b.Y / b.W);
    a.Y = sumY;
    if (std::fabs(a.Y) > kSmall) {
        Y1 /= a.Y;
        const double Y2 = b.Y / a.Y;
        a.Tlow = std::max(a.Tlow, b.Tlow);
        a.Thigh = std::min(a.Thigh, b.Thigh);
        for (int k = 0; k < 7; ++k) {
            a.high[k] = Y1 * a.high[k] + Y2 * b.high[k];
            a.low[k] = Y1 * a.low[k] + Y2 * b.low[k];
        }
    }
}

gf_thermo thermo_eq(const gf_thermo& t1, const gf_thermo& t2) {
    gf_thermo r;
    double diffY = t2.Y - t1.Y;
    if (std::fabs(diffY) < kSmall) diffY = kSmall;
    const double diffRW = t2.Y / t2.W - t1.Y / t1.W;
    double molWeight = kGreat;
    if (std::fabs(diffRW) > kSmall) molWeight = diffY / diffRW;
    r.Y = diffY;
    r.W = molWeight;
    const double Y1 = t2.Y / r.Y;
    const double Y2 = t1.Y / r.Y;
    for (int k = 0; k < 7; ++k) {
        r.high[k] = Y1 * t2.high[k] - Y2 * t1.high[k];
        r.low[k] = Y1 * t2.low[k] - Y2 * t1.low[k];
    }
    r.Tlow = std::max(t2.Tlow, t1.Tlow);
    r.Thigh = std::min(t2.Thigh, t1.Thigh);
    r.Tcommon = t2.Tcommon;
    return r;
}

gf_thermo thermo_scaled(const gf_thermo& t, double stoich) {
    gf_thermo r = t;
    r.Y = (stoich * t.W) * t.Y;
    return r;
}

bool valid_ptr(const void* p) { return p != nullptr; }

// ---- device buffer with sub-allocation

struct DevBuf {
    std::vector<char> host;
    size_t add(const void* src, size_t bytes) {
        const size_t off = (host.size() + 255) & ~size_t(255);
        host.resize(off + bytes);
        if (bytes) std::memcpy(host.data() + off, src, bytes);
        return off;
    }
    template <class T>
    size_t add(const std::vector<T>& v) {
        return add(v.data(), v.size() * sizeof(T));
    }
};

// Gather streams (gf::Stream): entries with their (slot, coef) records in
// summation order, split over G threads so that the record counts balance
// (greedy, largest entry first), each thread's entries in ascending order,
// interleaved record k of thread t at k * G + t, padded to the longest thread.
// An entry without records still gets one (it writes zero).
std::vector<gf::StreamRec> build_stream(const std::vector<std::vector<std::pair<int, double>>>& entries,
                                        const std::vector<int>& pos, int G, int* len_out) {
    const int nE = (int)entries.size();
    std::vector<int> order(nE);
    for (int e = 0; e < nE; ++e) order[e] = e;
    auto cnt = [&](int e) { return std::max<int>(1, (int)entries[e].size()); };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cnt(a) > cnt(b); });
    std::vector<long long> load(G, 0);
    std::vector<std::vector<int>> owned(G);
    for (int e : order) {
        int t = 0;
        for (int u = 1; u < G; ++u)
            if (load[u] < load[t]) t = u;
        load[t] += cnt(e);
        owned[t].push_back(e);
    }
    int len = 0;
    for (int t = 0; t < G; ++t) len = std::max<int>(len, (int)load[t]);
    std::vector<gf::StreamRec> rec((size_t)std::max(len, 1) * G, gf::StreamRec{-1, -1, 0.0});
    for (int t = 0; t < G; ++t) {
        std::sort(owned[t].begin(), owned[t].end());
        int k = 0;
        for (int e : owned[t]) {
            const auto& R = entries[e];
            if (R.empty()) {
                rec[(size_t)k++ * G + t] = gf::StreamRec{pos[e], -1, 0.0};
                continue;
            }
            for (size_t i = 0; i < R.size(); ++i)
                rec[(size_t)k++ * G + t] = gf::StreamRec{i + 1 == R.size() ? pos[e] : -1, R[i].first, R[i].second};
        }
    }
    *len_out = len;
    return rec;
}

}  // namespace

struct gf_mech {
    gf::DevMech dev;
    std::vector<int> q_of_r;  // compute position of each reaction (mechanism order)
    void* dmem = nullptr;
    long long bytes = 0;
    int device = 0;
};

struct gf_solver {
    std::vector<const gf_mech*> mechs;
    std::vector<gf::DevMech> dmechs;
    gf::OdeParams ode;
    double Treact = 0.0;
    gf_launch_config cfg;
    unsigned long long* queue = nullptr;  // device
    unsigned long long* queue_host = nullptr;  // pinned
    double* ws = nullptr;
    size_t ws_bytes = 0;
    double* adj_ws = nullptr;  // the adjoint sweep's workspaces
    size_t adj_ws_bytes = 0;
    int max_ws_doubles = 0;
    int max_neq = 0;
    // device staging for the host-memory entry points
    double* dY = nullptr;
    double* dYnew = nullptr;
    double* dRR = nullptr;
    double* drho = nullptr;
    double* ddtc = nullptr;
    double* ddt = nullptr;  // per-cell flow time steps (local time stepping)
    int staged_cells = 0;
};

namespace gf {
const DevMech* mech_device_tables(const gf_mech* m) { return &m->dev; }
int mech_device(const gf_mech* m) { return m->device; }
int record_cuda_error(int e) { return cuda_fail((cudaError_t)e); }
}  // namespace gf

namespace {

int ensure_ws(gf_solver* s, size_t bytes) {
    if (bytes <= s->ws_bytes) return GF_OK;
    if (s->ws) cudaFree(s->ws);
    s->ws = nullptr;
    s->ws_bytes = 0;
    GF_CUDA(cudaMalloc(&s->ws, bytes));
    s->ws_bytes = bytes;
    return GF_OK;
}

int ensure_staging(gf_solver* s, int n) {
    if (n <= s->staged_cells) return GF_OK;
    cudaFree(s->dY);
    cudaFree(s->dYnew);
    cudaFree(s->dRR);
    cudaFree(s->drho);
    cudaFree(s->ddtc);
    cudaFree(s->ddt);
    s->dY = s->dYnew = s->dRR = s->drho = s->ddtc = s->ddt = nullptr;
    s->staged_cells = 0;
    const size_t ne = (size_t)s->max_neq;
    GF_CUDA(cudaMalloc(&s->dY, (size_t)n * ne * sizeof(double)));
    GF_CUDA(cudaMalloc(&s->dYnew, (size_t)n * ne * sizeof(double)));
    GF_CUDA(cudaMalloc(&s->dRR, (size_t)n * ne * sizeof(double)));
    GF_CUDA(cudaMalloc(&s->drho, (size_t)n * sizeof(double)));
    GF_CUDA(cudaMalloc(&s->ddtc, (size_t)n * sizeof(double)));
    GF_CUDA(cudaMalloc(&s->ddt, (size_t)n * sizeof(double)));
    s->staged_cells = n;
    return GF_OK;
}

}  // namespace

extern "C" {

int gf_abi_version(void) { return GF_ABI_VERSION; }

const char* gf_last_cuda_error(void) { return g_last_cuda_error.c_str(); }

const char* gf_strerror(int status) {
    switch (status) {
    case GF_OK: return "ok";
    case GF_ERR_INVALID_ARGUMENT: return "invalid argument";
    case GF_ERR_UNKNOWN_SOLVER: return "Invalid ODE Solver type";
    case GF_ERR_UNSUPPORTED: return "mechanism outside the supported limits";
    case GF_ERR_MASS_IMBALANCE: return "mass imbalance in reaction (> 0.1 kg/kmol)";
    case GF_ERR_CUDA: return "CUDA runtime error";
    case GF_ERR_NO_DEVICE: return "no CUDA device";
    case GF_ERR_OUT_OF_MEMORY: return "out of device memory";
    case GF_ERR_CELL_FAILURE: return "one or more cells failed to integrate";
    default: return "unknown status";
    }
}

// makeGpuThermo (makeGpuThermo.H:16-48)
int gf_thermo_from_nasa(double Y, double W, double Tlow, double Thigh, double Tcommon, const double high_raw[7],
                        const double low_raw[7], gf_thermo* out) {
    if (!high_raw || !low_raw || !out || !(W > 0)) return GF_ERR_INVALID_ARGUMENT;
    const double R = kRR / W;  // specie gas constant, gpuPerfectGas.H:141-143
    out->Y = Y;
    out->W = W;
    out->Tlow = Tlow;
    out->Thigh = Thigh;
    out->Tcommon = Tcommon;
    for (int k = 0; k < 7; ++k) {
        out->high[k] = R * high_raw[k];
        out->low[k] = R * low_raw[k];
    }
    return GF_OK;
}

// set_reaction_thermo (makeGpuReactions.H:18-59)
int gf_reaction_thermo(const gf_thermo* species, int n_species, int n_lhs, const gf_specie_coeff* lhs, int n_rhs,
                       const gf_specie_coeff* rhs, gf_thermo* out) {
    if (!species || !lhs || !rhs || !out || n_lhs < 1 || n_rhs < 1) return GF_ERR_INVALID_ARGUMENT;
    for (int i = 0; i < n_lhs; ++i)
        if (lhs[i].index < 0 || lhs[i].index >= n_species) return GF_ERR_INVALID_ARGUMENT;
    for (int i = 0; i < n_rhs; ++i)
        if (rhs[i].index < 0 || rhs[i].index >= n_species) return GF_ERR_INVALID_ARGUMENT;
    gf_thermo r = thermo_scaled(species[rhs[0].index], rhs[0].stoich);
    for (int i = 1; i < n_rhs; ++i) thermo_add(r, thermo_scaled(species[rhs[i].index], rhs[i].stoich));
    gf_thermo l = thermo_scaled(species[lhs[0].index], lhs[0].stoich);
    for (int i = 1; i < n_lhs; ++i) thermo_add(l, thermo_scaled(species[lhs[i].index], lhs[i].stoich));
    if (std::fabs(l.Y - r.Y) > 0.1) return GF_ERR_MASS_IMBALANCE;
    *out = thermo_eq(l, r);
    return GF_OK;
}

int gf_mech_create(const gf_mech_desc* d, gf_mech** out) {
    if (!d || !out || !d->thermos || (d->n_reactions > 0 && !d->reactions)) return GF_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    const int nS = d->n_species, nR = d->n_reactions;
    if (nS < 1 || nR < 0) return GF_ERR_INVALID_ARGUMENT;
    if (nS > GF_MAX_SPECIES) return GF_ERR_UNSUPPORTED;
    using namespace gf;
    // ---- validation
    double Tlow = 0, Thigh = DBL_MAX / 10;
    if (!(nR >= 0)) return GF_ERR_INVALID_ARGUMENT;
    for (int r = 0; r < nR; ++r) {
        const gf_reaction& x = d->reactions[r];
        if (x.n_lhs < 1 || x.n_rhs < 1 || x.n_lhs > kMaxW || x.n_rhs > kMaxW) return GF_ERR_UNSUPPORTED;
        if (x.rate_type < 0 || x.rate_type > 3) return GF_ERR_INVALID_ARGUMENT;
        if (x.rate_type != GF_RATE_ARRHENIUS && !x.efficiencies) return GF_ERR_INVALID_ARGUMENT;
        for (int i = 0; i < x.n_lhs; ++i)
            if (x.lhs[i].index < 0 || x.lhs[i].index >= nS) return GF_ERR_INVALID_ARGUMENT;
        for (int i = 0; i < x.n_rhs; ++i)
            if (x.rhs[i].index < 0 || x.rhs[i].index >= nS) return GF_ERR_INVALID_ARGUMENT;
        // one set of limits per mechanism, as makeGpuReactions sets them (makeGpuReactions.H:121-124)
        if (r == 0) {
            Tlow = x.Tlow;
            Thigh = x.Thigh;
        } else if (x.Tlow != Tlow || x.Thigh != Thigh) {
            return GF_ERR_UNSUPPORTED;
        }
    }
    for (int i = 0; i < nS; ++i)
        if (!(d->thermos[i].W > 0)) return GF_ERR_INVALID_ARGUMENT;

    // ---- host tables
    std::vector<double> W(nS), Rsp(nS), Tc(nS), coef((size_t)14 * nS), hf(nS);
    for (int i = 0; i < nS; ++i) {
        const gf_thermo& t = d->thermos[i];
        W[i] = t.W;
        // enthalpy of formation, gpuThermo::Hf (gpuThermo.H:243-254), for Qdot
        const double* a = t.low;
        const double Ts = kTstd;
        hf[i] = (((((a[4] / 5.0 * Ts + a[3] / 4.0) * Ts + a[2] / 3.0) * Ts + a[1] / 2.0) * Ts + a[0]) * Ts + a[5]);
        Rsp[i] = kRR / t.W;
        Tc[i] = t.Tcommon;
        for (int k = 0; k < 7; ++k) {
            coef[(size_t)k * nS + i] = t.low[k];
            coef[(size_t)(7 + k) * nS + i] = t.high[k];
        }
    }
    const int nRa = std::max(nR, 1);
    // compute order: reactions grouped by rate type (stable within a type)
    std::vector<int> qof(nRa, 0), rof(nRa, 0);  // q -> r and r -> q
    {
        std::vector<int> o(nR);
        for (int r = 0; r < nR; ++r) o[r] = r;
        std::stable_sort(o.begin(), o.end(),
                         [&](int a, int b) { return d->reactions[a].rate_type < d->reactions[b].rate_type; });
        for (int q = 0; q < nR; ++q) {
            qof[q] = o[q];
            rof[o[q]] = q;
        }
    }
    std::vector<int> rtype(nRa), rirr(nRa), nl(nRa), nr(nRa), sp_off(nRa + 1, 0), slot(nRa + 1, 0),
        rnm_small(nRa), tb_row(nRa, -1);
    std::vector<double> rY(nRa), rnm(nRa), rTc(nRa), rcoef((size_t)14 * nRa), troe((size_t)4 * nRa, 0.0);
    std::vector<double> lnA0(nRa), sA0(nRa), beta0(nRa), Ta0(nRa), lnA1(nRa, 0.0), sA1(nRa, 0.0), beta1(nRa, 0.0),
        Ta1(nRa, 0.0);
    std::vector<int> sidx, siexp;
    std::vector<double> sst, sexp, eff;
    auto logabs = [](double A, double* lnA, double* sA) {
        // k = sign(A) exp(ln|A| + ...): A == 0 gives sign 0 (k == 0 exactly)
        *sA = A > 0 ? 1.0 : (A < 0 ? -1.0 : 0.0);
        *lnA = A != 0 ? std::log(std::fabs(A)) : 0.0;
    };
    int n_tb = 0;
    for (int q = 0; q < nR; ++q) {
        const gf_reaction& x = d->reactions[qof[q]];
        rtype[q] = x.rate_type;
        rirr[q] = x.irreversible ? 1 : 0;
        nl[q] = x.n_lhs;
        nr[q] = x.n_rhs;
        rY[q] = x.thermo.Y;
        const double nm = x.thermo.Y / x.thermo.W;
        rnm[q] = nm;
        rnm_small[q] = std::fabs(nm - kSmall) < kVSmall ? 1 : 0;  // gpuThermo.H:111, 146
        rTc[q] = x.thermo.Tcommon;
        for (int k = 0; k < 7; ++k) {
            rcoef[(size_t)k * nRa + q] = x.thermo.low[k];
            rcoef[(size_t)(7 + k) * nRa + q] = x.thermo.high[k];
        }
        logabs(x.A, &lnA0[q], &sA0[q]);
        beta0[q] = x.beta;
        Ta0[q] = x.Ta;
        if (x.rate_type == GF_RATE_LINDEMANN_FALLOFF || x.rate_type == GF_RATE_TROE_FALLOFF) {
            logabs(x.Ainf, &lnA1[q], &sA1[q]);
            beta1[q] = x.betainf;
            Ta1[q] = x.Tainf;
        }
        troe[4 * q + 0] = x.troe_alpha;
        troe[4 * q + 1] = 1.0 / x.troe_Tsss;
        troe[4 * q + 2] = 1.0 / x.troe_Ts;
        troe[4 * q + 3] = x.troe_Tss;
        if (x.rate_type != GF_RATE_ARRHENIUS) {
            tb_row[q] = n_tb++;
            eff.insert(eff.end(), x.efficiencies, x.efficiencies + nS);
        }
        for (int e = 0; e < x.n_lhs + x.n_rhs; ++e) {
            const gf_specie_coeff& sc = e < x.n_lhs ? x.lhs[e] : x.rhs[e - x.n_lhs];
            sidx.push_back(sc.index);
            sst.push_back(sc.stoich);
            if (sc.integer_exponent) {
                siexp.push_back((int)sc.exponent);
                sexp.push_back((double)(int)sc.exponent);
            } else {
                siexp.push_back(kNoIntExp);
                sexp.push_back(sc.exponent);
            }
        }
        sp_off[q + 1] = sp_off[q] + x.n_lhs + x.n_rhs;
        slot[q + 1] = slot[q] + 2 + x.n_lhs + x.n_rhs + (x.rate_type == GF_RATE_THIRD_BODY_ARRHENIUS ? 1 : 0);
    }
    const int n_slots = slot[nR];
    // per-species terms, built over reactions in mechanism order r
    std::vector<std::vector<std::pair<int, double>>> dn(nS);
    const int nE = nS * (nS + 1);  // raw-Jacobian entries: species rows x (species + T) columns
    std::vector<std::vector<std::pair<int, double>>> je(nE);
    for (int r = 0; r < nR; ++r) {
        const gf_reaction& x = d->reactions[r];
        const int so = slot[rof[r]];
        // dNdtByV (gpuReaction.H:490-508)
        for (int i = 0; i < x.n_lhs; ++i) dn[x.lhs[i].index].push_back({so, -x.lhs[i].stoich});
        for (int i = 0; i < x.n_rhs; ++i) dn[x.rhs[i].index].push_back({so, x.rhs[i].stoich});
        auto add = [&](int s, int c, int sl, double cf) { je[(size_t)s * (nS + 1) + c].push_back({sl, cf}); };
        // jac_dCfdcj_contribution (gpuReaction.H:547-569)
        for (int j = 0; j < x.n_lhs; ++j) {
            const int sj = x.lhs[j].index;
            for (int i = 0; i < x.n_lhs; ++i) add(x.lhs[i].index, sj, so + 2 + j, -x.lhs[i].stoich);
            for (int i = 0; i < x.n_rhs; ++i) add(x.rhs[i].index, sj, so + 2 + j, x.rhs[i].stoich);
        }
        // jac_dCrdcj_contribution (:571-593); an irreversible reaction adds zeros
        if (!x.irreversible) {
            for (int j = 0; j < x.n_rhs; ++j) {
                const int sj = x.rhs[j].index;
                for (int i = 0; i < x.n_lhs; ++i) add(x.lhs[i].index, sj, so + 2 + x.n_lhs + j, x.lhs[i].stoich);
                for (int i = 0; i < x.n_rhs; ++i) add(x.rhs[i].index, sj, so + 2 + x.n_lhs + j, -x.rhs[i].stoich);
            }
        }
        // jac_dCdT_contribution (:595-612)
        for (int i = 0; i < x.n_lhs; ++i) add(x.lhs[i].index, nS, so + 1, -x.lhs[i].stoich);
        for (int i = 0; i < x.n_rhs; ++i) add(x.rhs[i].index, nS, so + 1, x.rhs[i].stoich);
        // jac_dCdC_contribution (:614-648): fall-off ddc is identically zero (kInf
        // has no concentration dependence, gpuFallOffReactionRate.H:143-153)
        if (x.rate_type == GF_RATE_THIRD_BODY_ARRHENIUS) {
            const int sp = so + 2 + x.n_lhs + x.n_rhs;  // Ak * (Cf - Cr/Kc)
            for (int i = 0; i < x.n_lhs; ++i)
                for (int c = 0; c < nS; ++c) add(x.lhs[i].index, c, sp, -x.lhs[i].stoich * x.efficiencies[c]);
            for (int i = 0; i < x.n_rhs; ++i)
                for (int c = 0; c < nS; ++c) add(x.rhs[i].index, c, sp, x.rhs[i].stoich * x.efficiencies[c]);
        }
    }
    std::vector<RxnHead> rxh(nRa);
    std::vector<RxnSpecie> rxs((size_t)nRa * 2 * kSideInline, RxnSpecie{0, 1, 1.0});
    for (int q = 0; q < nR; ++q) {
        RxnHead& h = rxh[q];
        h.type = rtype[q];
        h.irr = rirr[q];
        h.slot = slot[q];
        h.tb_row = tb_row[q];
        h.nl = nl[q];
        h.nr = nr[q];
        h.sp_off = sp_off[q];
        h.nm_small = rnm_small[q];
        h.lnA0 = lnA0[q];
        h.beta0 = beta0[q];
        h.Ta0 = Ta0[q];
        h.sA0 = sA0[q];
        h.Tcommon = rTc[q];
        h.Y = rY[q];
        h.nm = rnm[q];
        h.pad = 0.0;
        for (int side = 0; side < 2; ++side) {
            const int n = side == 0 ? nl[q] : nr[q];
            const int b = sp_off[q] + (side == 0 ? 0 : nl[q]);
            for (int e = 0; e < n && e < kSideInline; ++e)
                rxs[((size_t)q * 2 + side) * kSideInline + e] = RxnSpecie{sidx[b + e], siexp[b + e], sexp[b + e]};
        }
    }
    const int ldJ = (nS + 1) | 1;  // the workspace Jacobian row stride (make_layout)
    std::vector<int> dn_pos(nS), je_pos(nE);
    for (int s2 = 0; s2 < nS; ++s2) dn_pos[s2] = s2;
    for (int e = 0; e < nE; ++e) je_pos[e] = (e / (nS + 1)) * ldJ + e % (nS + 1);
    // concentration gathers of the adjoint: species s <- entry slots of its occurrences
    std::vector<std::vector<std::pair<int, double>>> cg(nS);
    int max_side = 0;
    for (int q = 0; q < nR; ++q) {
        max_side = std::max(max_side, std::max(nl[q], nr[q]));
        for (int side = 0; side < 2; ++side) {
            const int n = side == 0 ? nl[q] : nr[q];
            const int b = sp_off[q] + (side == 0 ? 0 : nl[q]);
            for (int e = 0; e < n && e < kSideInline; ++e)
                cg[sidx[b + e]].push_back({q * 2 * kSideInline + side * kSideInline + e, 1.0});
        }
    }
    std::vector<std::vector<StreamRec>> dst_rec(kNumGroupSizes), jst_rec(kNumGroupSizes), cst_rec(kNumGroupSizes);
    int dst_len[kNumGroupSizes], jst_len[kNumGroupSizes], cst_len[kNumGroupSizes];
    for (int k = 0; k < kNumGroupSizes; ++k) {
        dst_rec[k] = build_stream(dn, dn_pos, group_size_of(k), &dst_len[k]);
        jst_rec[k] = build_stream(je, je_pos, group_size_of(k), &jst_len[k]);
        cst_rec[k] = build_stream(cg, dn_pos, group_size_of(k), &cst_len[k]);
    }
    // keep every array non-empty
    if (eff.empty()) eff.push_back(0.0);
    if (sidx.empty()) {
        sidx.push_back(0);
        siexp.push_back(0);
        sst.push_back(0.0);
        sexp.push_back(0.0);
    }

    // ---- every index the kernels follow, checked before upload: a table that
    // would send a kernel outside its arrays is refused here, not found on the GPU
    {
        const int m = nS + 1;
        auto stream_ok = [](const std::vector<StreamRec>& rec, int n_pos, int n_src) {
            for (const StreamRec& r : rec)
                if (r.pos >= n_pos || r.slot >= n_src) return false;
            return true;
        };
        const int n_conc_slots = 2 * kSideInline * nRa;
        for (int k = 0; k < kNumGroupSizes; ++k)
            if (!stream_ok(dst_rec[k], nS, n_slots) || !stream_ok(jst_rec[k], m * ldJ, n_slots) ||
                !stream_ok(cst_rec[k], nS, n_conc_slots))
                return GF_ERR_UNSUPPORTED;
        for (int q = 0; q < nR; ++q) {
            const int need = std::max(4, 2 + nl[q] + nr[q] + (rtype[q] == GF_RATE_THIRD_BODY_ARRHENIUS ? 1 : 0));
            if (slot[q] < 0 || slot[q] + need > n_slots) return GF_ERR_UNSUPPORTED;
            if (tb_row[q] >= n_tb || (rtype[q] != GF_RATE_ARRHENIUS && tb_row[q] < 0)) return GF_ERR_UNSUPPORTED;
            if (sp_off[q] < 0 || (size_t)sp_off[q] + nl[q] + nr[q] > sidx.size()) return GF_ERR_UNSUPPORTED;
            for (int e = 0; e < nl[q] + nr[q]; ++e)
                if (sidx[sp_off[q] + e] < 0 || sidx[sp_off[q] + e] >= nS) return GF_ERR_UNSUPPORTED;
        }
        if (eff.size() < (size_t)std::max(n_tb, 1) * (n_tb > 0 ? nS : 1)) return GF_ERR_UNSUPPORTED;
    }

    // ---- one device allocation
    DevBuf b;
    const size_t oW = b.add(W), oR = b.add(Rsp), oTc = b.add(Tc), oCoef = b.add(coef), oHf = b.add(hf);
    const size_t oRt = b.add(rtype), oRi = b.add(rirr), oNl = b.add(nl), oNr = b.add(nr), oSpo = b.add(sp_off),
                 oSlot = b.add(slot), oRY = b.add(rY), oRnm = b.add(rnm), oRns = b.add(rnm_small), oRTc = b.add(rTc),
                 oRc = b.add(rcoef), oLA0 = b.add(lnA0), oSA0 = b.add(sA0), oB0 = b.add(beta0), oT0 = b.add(Ta0),
                 oLA1 = b.add(lnA1), oSA1 = b.add(sA1), oB1 = b.add(beta1), oT1 = b.add(Ta1), oTroe = b.add(troe),
                 oTb = b.add(tb_row), oEff = b.add(eff), oSi = b.add(sidx), oSie = b.add(siexp), oSst = b.add(sst),
                 oSe = b.add(sexp), oRxh = b.add(rxh), oRxs = b.add(rxs), oRofq = b.add(qof);
    size_t oDst[kNumGroupSizes], oJst[kNumGroupSizes], oCst[kNumGroupSizes];
    for (int k = 0; k < kNumGroupSizes; ++k) {
        oDst[k] = b.add(dst_rec[k]);
        oJst[k] = b.add(jst_rec[k]);
        oCst[k] = b.add(cst_rec[k]);
    }
    gf_mech* m = new (std::nothrow) gf_mech;
    if (!m) return GF_ERR_OUT_OF_MEMORY;
    cudaGetDevice(&m->device);
    cudaError_t e = cudaMalloc(&m->dmem, b.host.size());
    if (e != cudaSuccess) {
        delete m;
        return cuda_fail(e);
    }
    e = cudaMemcpy(m->dmem, b.host.data(), b.host.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(m->dmem);
        delete m;
        return cuda_fail(e);
    }
    m->bytes = (long long)b.host.size();
    char* base = static_cast<char*>(m->dmem);
    auto P = [&](size_t o) { return base + o; };
    DevMech& D = m->dev;
    D.nS = nS;
    D.nR = nR;
    D.m = nS + 1;
    D.n_slots = n_slots;
    D.n_tb = n_tb;
    D.Tlow = Tlow;
    D.Thigh = Thigh;
    D.W = (const double*)P(oW);
    D.Rsp = (const double*)P(oR);
    D.Tcommon = (const double*)P(oTc);
    D.coef = (const double*)P(oCoef);
    D.hf = (const double*)P(oHf);
    D.rtype = (const int*)P(oRt);
    D.rirr = (const int*)P(oRi);
    D.nl = (const int*)P(oNl);
    D.nr = (const int*)P(oNr);
    D.sp_off = (const int*)P(oSpo);
    D.slot = (const int*)P(oSlot);
    D.rY = (const double*)P(oRY);
    D.rnm = (const double*)P(oRnm);
    D.rnm_small = (const int*)P(oRns);
    D.rTcommon = (const double*)P(oRTc);
    D.rcoef = (const double*)P(oRc);
    D.lnA0 = (const double*)P(oLA0);
    D.sA0 = (const double*)P(oSA0);
    D.beta0 = (const double*)P(oB0);
    D.Ta0 = (const double*)P(oT0);
    D.lnA1 = (const double*)P(oLA1);
    D.sA1 = (const double*)P(oSA1);
    D.beta1 = (const double*)P(oB1);
    D.Ta1 = (const double*)P(oT1);
    D.troe = (const double*)P(oTroe);
    D.tb_row = (const int*)P(oTb);
    D.eff = (const double*)P(oEff);
    D.r_of_q = (const int*)P(oRofq);
    D.rxh = (const RxnHead*)P(oRxh);
    D.rxs = (const RxnSpecie*)P(oRxs);
    D.sidx = (const int*)P(oSi);
    D.siexp = (const int*)P(oSie);
    D.sst = (const double*)P(oSst);
    D.sexp = (const double*)P(oSe);
    for (int k = 0; k < kNumGroupSizes; ++k) {
        D.dst[k] = Stream{(const StreamRec*)P(oDst[k]), dst_len[k]};
        D.jst[k] = Stream{(const StreamRec*)P(oJst[k]), jst_len[k]};
        D.cst[k] = Stream{(const StreamRec*)P(oCst[k]), cst_len[k]};
    }
    D.max_side = max_side;
    m->q_of_r.assign(rof.begin(), rof.begin() + nR);
    *out = m;
    return GF_OK;
}

void gf_mech_destroy(gf_mech* m) {
    if (!m) return;
    if (m->dmem) cudaFree(m->dmem);
    delete m;
}

int gf_mech_info(const gf_mech* m, int* n_species, int* n_reactions, long long* device_bytes) {
    if (!m) return GF_ERR_INVALID_ARGUMENT;
    if (n_species) *n_species = m->dev.nS;
    if (n_reactions) *n_reactions = m->dev.nR;
    if (device_bytes) *device_bytes = m->bytes;
    return GF_OK;
}

int gf_solver_create(const gf_mech* const* mechs, int n_mechs, const gf_ode_inputs* in, double Treact,
                     gf_solver** out) {
    if (!mechs || n_mechs < 1 || n_mechs > 4 || !in || !out) return GF_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    // make_gpuODESolver (makeGpuOdeSolver.H:13-31)
    if (in->solver != GF_ROSENBROCK12 && in->solver != GF_ROSENBROCK23 && in->solver != GF_ROSENBROCK34)
        return GF_ERR_UNKNOWN_SOLVER;
    if (in->maxSteps < 0) return GF_ERR_INVALID_ARGUMENT;
    for (int i = 0; i < n_mechs; ++i)
        if (!mechs[i]) return GF_ERR_INVALID_ARGUMENT;
    gf_solver* s = new (std::nothrow) gf_solver;
    if (!s) return GF_ERR_OUT_OF_MEMORY;
    for (int i = 0; i < n_mechs; ++i) {
        s->mechs.push_back(mechs[i]);
        s->dmechs.push_back(mechs[i]->dev);
        s->max_ws_doubles = std::max(s->max_ws_doubles, gf::ws_layout(mechs[i]->dev).size);
        s->max_neq = std::max(s->max_neq, mechs[i]->dev.nS + 2);
    }
    s->ode = gf::OdeParams{in->solver, in->absTol, in->relTol, in->maxSteps, in->safeScale, in->alphaInc,
                           in->alphaDec, in->minScale, in->maxScale};
    s->Treact = Treact;
    // default launch: persistent, two warps per cell (one cell per CTA),
    // workspace in shared memory when it fits (the autotuner refines this per
    // mechanism)
    s->cfg = gf_launch_config{1, 64, 1, 1, 0, 0, 0, 0};  // kind, G, shared, cells/CTA, CTAs/SM, registers, panel, specialize
    if ((size_t)s->max_ws_doubles * sizeof(double) > 227 * 1024) s->cfg.scratch_in_shared = 0;
    cudaError_t e = cudaMalloc(&s->queue, 8 * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMallocHost(&s->queue_host, 8 * sizeof(unsigned long long));
    if (e != cudaSuccess) {
        gf_solver_destroy(s);
        return cuda_fail(e);
    }
    *out = s;
    return GF_OK;
}

void gf_solver_destroy(gf_solver* s) {
    if (!s) return;
    cudaFree(s->queue);
    if (s->queue_host) cudaFreeHost(s->queue_host);
    cudaFree(s->ws);
    cudaFree(s->adj_ws);
    cudaFree(s->dY);
    cudaFree(s->dYnew);
    cudaFree(s->dRR);
    cudaFree(s->drho);
    cudaFree(s->ddtc);
    cudaFree(s->ddt);
    delete s;
}

int gf_solver_set_launch(gf_solver* s, const gf_launch_config* cfg) {
    if (!s || !cfg) return GF_ERR_INVALID_ARGUMENT;
    if (cfg->kind != 0 && cfg->kind != 1) return GF_ERR_INVALID_ARGUMENT;
    if (cfg->kind == 1) {
        const int G = cfg->threads_per_cell;
        if (G != 1 && G != 2 && G != 4 && G != 8 && G != 16 && G != 32 && G != 64 && G != 96 && G != 128 && G != 256)
            return GF_ERR_INVALID_ARGUMENT;
        if (cfg->register_budget != 0 && cfg->register_budget != 1) return GF_ERR_INVALID_ARGUMENT;
        if (cfg->scratch_in_shared && (size_t)s->max_ws_doubles * sizeof(double) > 227 * 1024)
            return GF_ERR_UNSUPPORTED;
        if (cfg->lu_panel != 0 && cfg->lu_panel != 4 && cfg->lu_panel != 8 && cfg->lu_panel != 16)
            return GF_ERR_INVALID_ARGUMENT;
        if (cfg->specialize != 0 && cfg->specialize != 1) return GF_ERR_INVALID_ARGUMENT;
        // the tuned variants (lu_panel 4 / 16, specialize) exist for some forms
        // only (gf_persist.cuh, persistent_tuned_variant)
        if (!gf::persistent_form_compiled(*cfg, gf::specialized_size(s->dmechs.data(), (int)s->dmechs.size())))
            return GF_ERR_UNSUPPORTED;
    }
    s->cfg = *cfg;
    return GF_OK;
}

int gf_solver_info(const gf_solver* s, int* ws_doubles_per_cell, int* max_neq, int* n_mechs) {
    if (!s) return GF_ERR_INVALID_ARGUMENT;
    if (ws_doubles_per_cell) *ws_doubles_per_cell = s->max_ws_doubles;
    if (max_neq) *max_neq = s->max_neq;
    if (n_mechs) *n_mechs = (int)s->mechs.size();
    return GF_OK;
}

int gf_solver_get_launch(const gf_solver* s, gf_launch_config* cfg) {
    if (!s || !cfg) return GF_ERR_INVALID_ARGUMENT;
    *cfg = s->cfg;
    return GF_OK;
}

}  // extern "C"

namespace {

// Arguments of one solve, checked; queue and workspace left for the caller.
int solve_args(const gf_solver* s, int n_cells, double deltaT, const double* deltaT_cell, double deltaTChemMax,
               const int* mech_id, const double* rho, const double* Y0, int ld_y, double* Ynew,
               double* deltaTChem, double* RR, int ld_rr, int* status, int* counters, gf::LaunchArgs* a) {
    if (!s || n_cells < 0 || !deltaTChem || !Y0) return GF_ERR_INVALID_ARGUMENT;
    if (ld_y < s->max_neq) return GF_ERR_INVALID_ARGUMENT;
    if (RR && (!rho || ld_rr < 1)) return GF_ERR_INVALID_ARGUMENT;
    if (!mech_id && s->mechs.size() > 1) return GF_ERR_INVALID_ARGUMENT;
    if (RR)
        for (const gf::DevMech& m : s->dmechs)
            if (ld_rr < m.nS) return GF_ERR_INVALID_ARGUMENT;  // every cell's row must hold its species
    a->n_cells = n_cells;
    a->deltaT = deltaT;
    a->deltaT_cell = deltaT_cell;
    a->deltaTChemMax = deltaTChemMax;
    a->mech_id = mech_id;
    a->rho = rho;
    a->Y0 = Y0;
    a->ld_y = ld_y;
    a->Ynew = Ynew;
    a->deltaTChem = deltaTChem;
    a->RR = RR;
    a->ld_rr = ld_rr;
    a->status = status;
    a->counters = counters;
    a->Treact = s->Treact;
    a->ode = s->ode;
    a->queue = nullptr;
    a->ws = nullptr;
    a->ws_slot_stride = 0;
    return GF_OK;
}

// Workspace slots (cells in flight with their workspace in HBM) of the
// solver's launch form for n_cells; 0 when the workspaces sit in shared memory.
int solve_slots(const gf_solver* s, int n_cells, int* slots) {
    *slots = 0;
    if (s->cfg.kind == 0) {
        *slots = n_cells;
        return GF_OK;
    }
    int blocks = 0, threads = 0;
    const int ms = gf::specialized_size(s->dmechs.data(), (int)s->dmechs.size());
    const int k = gf::persistent_slots(s->cfg, ms, s->max_ws_doubles * (int)sizeof(double), &blocks, &threads);
    if (k <= 0) return GF_ERR_UNSUPPORTED;
    if (!s->cfg.scratch_in_shared) *slots = k;
    return GF_OK;
}

double min_delta_t_of(unsigned long long k) {
    const unsigned long long bits = (k >> 63) ? (k & 0x7FFFFFFFFFFFFFFFull) : ~k;
    double mn;
    std::memcpy(&mn, &bits, 8);
    return mn;
}

void stats_of(const unsigned long long* q, int n_cells, gf_stats* stats) {
    stats->min_delta_t = n_cells > 0 ? min_delta_t_of(q[1]) : 0.0;
    stats->accepted_steps = (long long)q[2];
    stats->attempts = (long long)q[3];
    stats->failed_cells = (long long)q[4];
}

}  // namespace

extern "C" {

int gf_solve(gf_solver* s, int n_cells, double deltaT, const double* deltaT_cell, double deltaTChemMax,
             const int* mech_id, const double* rho, const double* Y0, int ld_y, double* Ynew, double* deltaTChem,
             double* RR, int ld_rr, int* status, int* counters, gf_stats* stats, void* stream) {
    gf::LaunchArgs a;
    int r = solve_args(s, n_cells, deltaT, deltaT_cell, deltaTChemMax, mech_id, rho, Y0, ld_y, Ynew, deltaTChem,
                       RR, ld_rr, status, counters, &a);
    if (r) return r;
    const int wsd = s->max_ws_doubles;
    int slots = 0;
    if ((r = solve_slots(s, n_cells, &slots))) return r;
    if (slots > 0 && (r = ensure_ws(s, (size_t)slots * wsd * sizeof(double)))) return r;
    a.queue = s->queue;
    a.ws = s->ws;
    a.ws_slot_stride = s->cfg.kind == 0 ? n_cells : 0;
    const int ce = gf::launch_cells(s->dmechs.data(), (int)s->dmechs.size(), s->cfg, a, wsd, slots, stream);
    if (ce) return cuda_fail((cudaError_t)ce);
    if (stats) {
        cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
        GF_CUDA(cudaMemcpyAsync(s->queue_host, s->queue, 5 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
        GF_CUDA(cudaStreamSynchronize(st));
        stats_of(s->queue_host, n_cells, stats);
    }
    return GF_OK;
}

// ---- graph-captured solve -----------------------------------------------------

}  // extern "C"

struct gf_solve_graph {
    gf_solver* solver = nullptr;
    gf_launch_config cfg{};                 // the launch form at capture time
    gf::LaunchArgs args{};
    int slots = 0;
    double* ws = nullptr;                   // the graph's own workspaces (HBM form)
    unsigned long long* queue = nullptr;    // its own work queue and step totals
    unsigned long long* queue_host = nullptr;
    cudaStream_t capture = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace {

// Records the queue reset, the solve kernel and the copy of the step totals
// to pinned host memory on the graph's private stream.
int capture_solve(gf_solve_graph* g, cudaGraph_t* out) {
    gf_solver* s = g->solver;
    GF_CUDA(cudaStreamBeginCapture(g->capture, cudaStreamCaptureModeRelaxed));
    int ce = gf::launch_cells(s->dmechs.data(), (int)s->dmechs.size(), g->cfg, g->args, s->max_ws_doubles,
                              g->slots, g->capture);
    if (!ce)
        ce = (int)cudaMemcpyAsync(g->queue_host, g->queue, 5 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                  g->capture);
    cudaGraph_t graph = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(g->capture, &graph);
    if (ce || ee) {
        if (graph) cudaGraphDestroy(graph);
        return cuda_fail(ce ? (cudaError_t)ce : ee);
    }
    *out = graph;
    return GF_OK;
}

}  // namespace

extern "C" {

int gf_solve_graph_create(gf_solver* s, int n_cells, double deltaT, const double* deltaT_cell,
                          double deltaTChemMax, const int* mech_id, const double* rho, const double* Y0, int ld_y,
                          double* Ynew, double* deltaTChem, double* RR, int ld_rr, int* status, int* counters,
                          gf_solve_graph** out) {
    if (!out) return GF_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    gf::LaunchArgs a;
    int r = solve_args(s, n_cells, deltaT, deltaT_cell, deltaTChemMax, mech_id, rho, Y0, ld_y, Ynew, deltaTChem,
                       RR, ld_rr, status, counters, &a);
    if (r) return r;
    auto* g = new gf_solve_graph;
    g->solver = s;
    g->cfg = s->cfg;
    g->args = a;
    const size_t wsd = (size_t)s->max_ws_doubles;
    if ((r = solve_slots(s, n_cells, &g->slots))) {
        delete g;
        return r;
    }
    cudaError_t e = cudaMalloc(&g->queue, 8 * sizeof(unsigned long long));
    if (!e) e = cudaMallocHost(&g->queue_host, 8 * sizeof(unsigned long long));
    if (!e && g->slots > 0) e = cudaMalloc(&g->ws, (size_t)g->slots * wsd * sizeof(double));
    if (!e) e = cudaStreamCreateWithFlags(&g->capture, cudaStreamNonBlocking);
    if (e) {
        gf_solve_graph_destroy(g);
        return cuda_fail(e);
    }
    std::memset(g->queue_host, 0, 8 * sizeof(unsigned long long));
    g->args.queue = g->queue;
    g->args.ws = g->ws;
    g->args.ws_slot_stride = s->cfg.kind == 0 ? n_cells : 0;
    if ((r = capture_solve(g, &g->graph))) {
        gf_solve_graph_destroy(g);
        return r;
    }
    e = cudaGraphInstantiate(&g->exec, g->graph, 0);
    if (e) {
        gf_solve_graph_destroy(g);
        return cuda_fail(e);
    }
    *out = g;
    return GF_OK;
}

int gf_solve_graph_set_delta_t(gf_solve_graph* g, double deltaT) {
    if (!g) return GF_ERR_INVALID_ARGUMENT;
    const double old = g->args.deltaT;
    g->args.deltaT = deltaT;
    cudaGraph_t graph = nullptr;
    int r = capture_solve(g, &graph);
    if (r) {
        g->args.deltaT = old;
        return r;
    }
    cudaGraphExecUpdateResultInfo info;
    cudaError_t e = cudaGraphExecUpdate(g->exec, graph, &info);
    if (e) {
        // the topology is the same by construction; instantiate afresh if the
        // driver still refuses the in-place update
        (void)cudaGetLastError();
        cudaGraphExec_t exec = nullptr;
        e = cudaGraphInstantiate(&exec, graph, 0);
        if (e) {
            cudaGraphDestroy(graph);
            g->args.deltaT = old;
            return cuda_fail(e);
        }
        cudaGraphExecDestroy(g->exec);
        g->exec = exec;
    }
    cudaGraphDestroy(g->graph);
    g->graph = graph;
    return GF_OK;
}

int gf_solve_graph_launch(gf_solve_graph* g, void* stream) {
    if (!g) return GF_ERR_INVALID_ARGUMENT;
    GF_CUDA(cudaGraphLaunch(g->exec, reinterpret_cast<cudaStream_t>(stream)));
    return GF_OK;
}

int gf_solve_graph_stats(const gf_solve_graph* g, gf_stats* stats) {
    if (!g || !stats) return GF_ERR_INVALID_ARGUMENT;
    stats_of(g->queue_host, g->args.n_cells, stats);
    return GF_OK;
}

void gf_solve_graph_destroy(gf_solve_graph* g) {
    if (!g) return;
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    if (g->capture) cudaStreamDestroy(g->capture);
    cudaFree(g->ws);
    cudaFree(g->queue);
    if (g->queue_host) cudaFreeHost(g->queue_host);
    delete g;
}

// ---- the plugin's field gather and rate scatter (gf_fieldio.cu) --------------

int gf_gather_states(int n_cells, int n_species, const double* const* Y_fields, const double* T, const double* p,
                     double* y, int ld_y, void* stream) {
    if (n_cells < 0 || n_species < 1 || n_species > GF_MAX_SPECIES || ld_y < n_species + 2 || !Y_fields)
        return GF_ERR_INVALID_ARGUMENT;
    if (n_cells == 0) return GF_OK;
    if (!T || !p || !y) return GF_ERR_INVALID_ARGUMENT;
    for (int i = 0; i < n_species; ++i)
        if (!Y_fields[i]) return GF_ERR_INVALID_ARGUMENT;
    const int e = gf::launch_gather_states(n_cells, n_species, Y_fields, T, p, y, ld_y, stream);
    return e ? cuda_fail((cudaError_t)e) : GF_OK;
}

int gf_scatter_rates(int n_cells, int n_species, const double* RR, int ld_rr, double* const* RR_fields,
                     void* stream) {
    if (n_cells < 0 || n_species < 1 || n_species > GF_MAX_SPECIES || ld_rr < n_species || !RR_fields)
        return GF_ERR_INVALID_ARGUMENT;
    if (n_cells == 0) return GF_OK;
    if (!RR) return GF_ERR_INVALID_ARGUMENT;
    for (int i = 0; i < n_species; ++i)
        if (!RR_fields[i]) return GF_ERR_INVALID_ARGUMENT;
    const int e = gf::launch_scatter_rates(n_cells, n_species, RR, ld_rr, RR_fields, stream);
    return e ? cuda_fail((cudaError_t)e) : GF_OK;
}

// ---- the plugin's per-cell side paths (gf_fields.cu) --------------------------

int gf_cell_rates(const gf_mech* m, int n_cells, const double* rho, const double* y, int ld_y, double* RR,
                  int ld_rr, double* tc, void* stream) {
    if (!m || n_cells < 0 || (n_cells > 0 && (!rho || !y))) return GF_ERR_INVALID_ARGUMENT;
    if (ld_y < m->dev.nS + 2 || (RR && ld_rr < m->dev.nS)) return GF_ERR_INVALID_ARGUMENT;
    if (!RR && !tc) return GF_OK;
    gf::FieldArgs a{n_cells, rho, y, ld_y, RR, ld_rr, tc, -1, -1, nullptr};
    const int e = gf::launch_cell_fields(m->dev, a, stream);
    return e ? (e == (int)cudaErrorInvalidValue ? GF_ERR_UNSUPPORTED : cuda_fail((cudaError_t)e)) : GF_OK;
}

int gf_reaction_rates(const gf_mech* m, int n_cells, int reaction, const double* rho, const double* y, int ld_y,
                      double* omega, double* RR, int ld_rr, void* stream) {
    if (!m || n_cells < 0 || (n_cells > 0 && (!rho || !y))) return GF_ERR_INVALID_ARGUMENT;
    if (reaction < 0 || reaction >= m->dev.nR) return GF_ERR_INVALID_ARGUMENT;
    if (ld_y < m->dev.nS + 2 || (RR && ld_rr < m->dev.nS)) return GF_ERR_INVALID_ARGUMENT;
    if (!RR && !omega) return GF_OK;
    gf::FieldArgs a{n_cells, rho, y, ld_y, RR, ld_rr, nullptr, reaction, m->q_of_r[reaction], omega};
    const int e = gf::launch_cell_fields(m->dev, a, stream);
    return e ? (e == (int)cudaErrorInvalidValue ? GF_ERR_UNSUPPORTED : cuda_fail((cudaError_t)e)) : GF_OK;
}

int gf_qdot(const gf_mech* m, int n_cells, const double* RR, int ld_rr, double* qdot, void* stream) {
    if (!m || n_cells < 0 || (n_cells > 0 && (!RR || !qdot)) || ld_rr < m->dev.nS) return GF_ERR_INVALID_ARGUMENT;
    const int e = gf::launch_qdot(m->dev, n_cells, RR, ld_rr, qdot, stream);
    return e ? cuda_fail((cudaError_t)e) : GF_OK;
}

// gf_solve with the trajectory recorded for the adjoint (single mechanism).
int gf_solve_record(gf_solver* s, int n_cells, double deltaT, const double* Y0, int ld_y, double* Ynew,
                    double* deltaTChem, int* status, int* counters, double* traj, int traj_cap, void* stream) {
    if (!s || n_cells < 0 || !Y0 || !Ynew || !deltaTChem || !status || !counters || !traj || traj_cap < 1)
        return GF_ERR_INVALID_ARGUMENT;
    if (s->mechs.size() != 1 || ld_y < s->max_neq) return GF_ERR_INVALID_ARGUMENT;
    gf::LaunchArgs a;
    a.n_cells = n_cells;
    a.deltaT = deltaT;
    a.deltaT_cell = nullptr;
    a.deltaTChemMax = INFINITY;
    a.mech_id = nullptr;
    a.rho = nullptr;
    a.Y0 = Y0;
    a.ld_y = ld_y;
    a.Ynew = Ynew;
    a.deltaTChem = deltaTChem;
    a.RR = nullptr;
    a.ld_rr = 0;
    a.status = status;
    a.counters = counters;
    a.Treact = s->Treact;
    a.ode = s->ode;
    a.queue = s->queue;
    a.traj = traj;
    a.traj_cap = traj_cap;
    a.traj_ld = s->dmechs[0].m + 1;
    a.ws = nullptr;
    a.ws_slot_stride = 0;
    const int ce = gf::launch_record(s->dmechs[0], a, stream);
    return ce ? (ce == (int)cudaErrorInvalidValue ? GF_ERR_UNSUPPORTED : cuda_fail((cudaError_t)ce)) : GF_OK;
}

// The reverse sweep over a recorded trajectory (gf_adjoint.cu).
int gf_adjoint(gf_solver* s, int n_cells, const double* traj, int traj_cap, const int* counters,
               const int* fwd_status, const double* Y0, const double* Ynew, const double* Ybar, int ld_y,
               double* Y0bar, double* theta_bar, int* status, void* stream) {
    if (!s || n_cells < 0 || !traj || traj_cap < 1 || !counters || !fwd_status || !Y0 || !Ynew || !Ybar ||
        !Y0bar || !theta_bar || !status)
        return GF_ERR_INVALID_ARGUMENT;
    if (s->mechs.size() != 1 || ld_y < s->max_neq) return GF_ERR_INVALID_ARGUMENT;
    const gf::DevMech& M = s->dmechs[0];
    if (M.max_side > gf::kSideInline) return GF_ERR_UNSUPPORTED;
    const int per_sm = gf::adjoint_blocks_per_sm(M);
    if (per_sm < 1) return GF_ERR_CUDA;
    const int blocks = per_sm * gf::device_sm_count();
    const long long wsd = gf::adjoint_ws_doubles(M);
    const size_t bytes = (size_t)blocks * wsd * sizeof(double);
    if (bytes > s->adj_ws_bytes) {
        cudaFree(s->adj_ws);
        s->adj_ws = nullptr;
        s->adj_ws_bytes = 0;
        GF_CUDA(cudaMalloc(&s->adj_ws, bytes));
        s->adj_ws_bytes = bytes;
    }
    const int e = gf::launch_adjoint_cells(M, n_cells, traj, traj_cap, counters, fwd_status, Y0, Ynew, Ybar, ld_y,
                                           Y0bar, theta_bar, status, s->ode, s->adj_ws, wsd, blocks, s->queue,
                                           stream);
    return e ? cuda_fail((cudaError_t)e) : GF_OK;
}

static int host_solve(gf_solver* s, int n, double deltaT, const double* deltaT_cell, double deltaTChemMax,
                      const double* rho, const double* deltaTChem, const double* Y, double* Ynew_out, double* RR_out,
                      double* deltaTChemNew, double* minDeltaT) {
    if (!s || n < 0 || !deltaTChem || !Y || !deltaTChemNew || s->mechs.size() != 1) return GF_ERR_INVALID_ARGUMENT;
    if (n == 0) return GF_OK;
    int r = ensure_staging(s, n);
    if (r) return r;
    const int ne = s->dmechs[0].nS + 2, nS = s->dmechs[0].nS;
    GF_CUDA(cudaMemcpyAsync(s->dY, Y, (size_t)n * ne * sizeof(double), cudaMemcpyHostToDevice, 0));
    GF_CUDA(cudaMemcpyAsync(s->ddtc, deltaTChem, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, 0));
    if (RR_out) GF_CUDA(cudaMemcpyAsync(s->drho, rho, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, 0));
    if (deltaT_cell)
        GF_CUDA(cudaMemcpyAsync(s->ddt, deltaT_cell, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, 0));
    gf_stats st;
    r = gf_solve(s, n, deltaT, deltaT_cell ? s->ddt : nullptr, deltaTChemMax, nullptr, RR_out ? s->drho : nullptr,
                 s->dY, ne, s->dYnew, s->ddtc, RR_out ? s->dRR : nullptr, nS, nullptr, nullptr, &st, 0);
    if (r) return r;
    if (Ynew_out) GF_CUDA(cudaMemcpy(Ynew_out, s->dYnew, (size_t)n * ne * sizeof(double), cudaMemcpyDeviceToHost));
    if (RR_out) GF_CUDA(cudaMemcpy(RR_out, s->dRR, (size_t)n * nS * sizeof(double), cudaMemcpyDeviceToHost));
    GF_CUDA(cudaMemcpy(deltaTChemNew, s->ddtc, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost));
    if (minDeltaT) *minDeltaT = st.min_delta_t;
    return GF_OK;
}

// GpuKernelEvaluator::computeRR (gpuKernelEvaluator.cu:65-97)
int gf_compute_rr(gf_solver* s, int n, double deltaT, double deltaTChemMax, const double* rho,
                  const double* deltaTChem, const double* Y, double* RR, double* deltaTChemNew, double* minDeltaT) {
    if (!rho || !RR) return GF_ERR_INVALID_ARGUMENT;
    return host_solve(s, n, deltaT, nullptr, deltaTChemMax, rho, deltaTChem, Y, nullptr, RR, deltaTChemNew,
                      minDeltaT);
}

// computeRR with a flow time step per cell: the local time stepping that
// gpuChemistryModel::solve(const scalarField&) rejects (gpuChemistryModel.C:328-333).
int gf_compute_rr_lts(gf_solver* s, int n, const double* deltaT, double deltaTChemMax, const double* rho,
                      const double* deltaTChem, const double* Y, double* RR, double* deltaTChemNew,
                      double* minDeltaT) {
    if (!rho || !RR || (n > 0 && !deltaT)) return GF_ERR_INVALID_ARGUMENT;
    return host_solve(s, n, 0.0, deltaT, deltaTChemMax, rho, deltaTChem, Y, nullptr, RR, deltaTChemNew, minDeltaT);
}

// GpuKernelEvaluator::computeYNew (gpuKernelEvaluator.cu:35-63): deltaTChemNew unclamped
int gf_compute_ynew(gf_solver* s, int n, double deltaT, double deltaTChemMax, const double* deltaTChem,
                    const double* Y, double* Ynew, double* deltaTChemNew) {
    (void)deltaTChemMax;
    if (!Ynew) return GF_ERR_INVALID_ARGUMENT;
    return host_solve(s, n, deltaT, nullptr, INFINITY, nullptr, deltaTChem, Y, Ynew, nullptr, deltaTChemNew,
                      nullptr);
}

int gf_rates(const gf_mech* m, int n, const double* y, double* dydx, void* stream) {
    if (!m || n < 0 || (n > 0 && (!y || !dydx))) return GF_ERR_INVALID_ARGUMENT;
    if ((size_t)gf::ws_layout(m->dev).size * sizeof(double) > 227 * 1024) return GF_ERR_UNSUPPORTED;
    const int e = gf::launch_rates(m->dev, n, y, dydx, stream);
    return e ? cuda_fail((cudaError_t)e) : GF_OK;
}

int gf_jacobian(const gf_mech* m, int n, const double* y, double* dfdx, double* J, void* stream) {
    if (!m || n < 0 || (n > 0 && (!y || !dfdx || !J))) return GF_ERR_INVALID_ARGUMENT;
    if ((size_t)gf::ws_layout(m->dev).size * sizeof(double) > 227 * 1024) return GF_ERR_UNSUPPORTED;
    const int e = gf::launch_jacobian(m->dev, n, y, dfdx, J, nullptr, stream);
    return e ? cuda_fail((cudaError_t)e) : GF_OK;
}

int gf_lu_decompose(int n_mats, int m, double* A, int* pivots, void* stream) {
    if (n_mats < 0 || m < 1 || m > 160 || (n_mats > 0 && (!A || !pivots))) return GF_ERR_INVALID_ARGUMENT;
    const int e = gf::launch_lu(n_mats, m, A, pivots, nullptr, stream);
    return e ? cuda_fail((cudaError_t)e) : GF_OK;
}

int gf_lu_factor_solve(int n_mats, int m, double* A, int* pivots, double* b, int n_rhs, int threads_per_matrix,
                       int exact, void* stream) {
    const int G = threads_per_matrix;
    if (G != 1 && G != 4 && G != 8 && G != 16 && G != 32 && G != 64 && G != 96 && G != 128 && G != 256)
        return GF_ERR_INVALID_ARGUMENT;
    if (n_mats < 0 || m < 1 || m > 160 || n_rhs < 0 || (n_mats > 0 && (!A || !pivots || (n_rhs > 0 && !b))))
        return GF_ERR_INVALID_ARGUMENT;
    const int e = gf::launch_lu_form(n_mats, m, A, pivots, b, n_rhs, G, exact != 0, stream);
    return e ? cuda_fail((cudaError_t)e) : GF_OK;
}

int gf_lu_backsubstitute(int n_mats, int m, const double* LU, const int* pivots, double* b, void* stream) {
    if (n_mats < 0 || m < 1 || m > 160 || (n_mats > 0 && (!LU || !pivots || !b))) return GF_ERR_INVALID_ARGUMENT;
    const int e = gf::launch_lusolve(n_mats, m, LU, pivots, b, stream);
    return e ? cuda_fail((cudaError_t)e) : GF_OK;
}

}  // extern "C"
