/*
 * TEST INFRASTRUCTURE ONLY — plain-C restatement of gpuFoam's per-cell
 * chemistry algorithm, used as the CPU oracle for the CUDA kernels.
 * Never linked or called by the product. Parity of this file with the
 * reference is pinned by tests/test_oracle.py against oracle/_ref (the
 * reference compiled in place) and tests/golden/.
 *
 * Every function follows the reference's operation order (compile with
 * -ffp-contract=off) and cites the reference file:line it restates; paths are
 * relative to the gpuFoam repository, under gpu_chemistry/src/ unless noted.
 */
#include "gf_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* gpu_utils/common/gpu_constants.H:13-82 */
#define ORC_RR (6.02214e+26 * 1.38065e-23)
#define ORC_PSTD 1e5
#define ORC_TSTD 298.15
#define ORC_VGREAT (DBL_MAX / 10.0)
#define ORC_VSMALL DBL_MIN
#define ORC_SMALL DBL_EPSILON
#define ORC_GREAT (1.0 / ORC_SMALL)
#define ORC_LOGTEN 2.302585092994046
#define ORC_MAXW 10
#define ORC_INT_MAX_10 (2147483647 / 10) /* gpuLabelMax */

enum { CELL_OK = 0, CELL_STEP_UNDERFLOW = 1, CELL_MAX_STEPS = 2, CELL_NONFINITE = 3, CELL_SKIPPED = 4 };

typedef struct {
    double Y, W, Tlow, Thigh, Tcommon;
    double high[7], low[7];
} thermo_t;

typedef struct {
    int index;
    int is_int; /* gpuSpecieExponent::hasIntegerExponent */
    int iexp;
    double stoich;
    double sexp; /* scalarExponent_ */
} coeff_t;

typedef struct {
    thermo_t th;
    int nl, nr;
    coeff_t lhs[ORC_MAXW], rhs[ORC_MAXW];
    int type, irr;
    double A, beta, Ta, Ainf, betainf, Tainf;
    double alpha, Tsss, Ts, Tss;
    const double* eff;
    double Tlow, Thigh;
} rxn_t;

typedef struct {
    int nS, nR;
    thermo_t* th;
    rxn_t* rx;
    double* eff;
} mech_t;

/* ---------------------------------------------------------------- thermo */

/* gpuEquationOfState/gpuPerfectGas.H:141-152 */
static double eos_R(const thermo_t* t) { return ORC_RR / t->W; }
static double eos_rho(const thermo_t* t, double p, double T) { return p / (eos_R(t) * T); }

/* gpuThermo/gpuThermo.H:29-32 */
static const double* coeffs(const thermo_t* t, double T) { return T < t->Tcommon ? t->low : t->high; }

/* gpuThermo.H:177-184 (+ gpuPerfectGas::Cp == 0, gpuPerfectGas.H:173-177) */
static double th_Cp_a(double T, const double* a) {
    return ((((a[4] * T + a[3]) * T + a[2]) * T + a[1]) * T + a[0]) + 0.0;
}
/* gpuThermo.H:210-221 */
static double th_Ha_a(double T, const double* a) {
    return (((((a[4] / 5.0 * T + a[3] / 4.0) * T + a[2] / 3.0) * T + a[1] / 2.0) * T + a[0]) * T + a[5]) + 0.0;
}
/* gpuThermo.H:243-254 */
static double th_Hf(const thermo_t* t) {
    const double* a = t->low;
    const double T = ORC_TSTD;
    return (((((a[4] / 5.0 * T + a[3] / 4.0) * T + a[2] / 3.0) * T + a[1] / 2.0) * T + a[0]) * T + a[5]);
}
/* gpuThermo.H:261-271 with gpuPerfectGas::Sp (gpuPerfectGas.H:210-214) */
static double th_S(const thermo_t* t, double p, double T, double logT) {
    const double* a = coeffs(t, T);
    return ((((a[4] / 4.0 * T + a[3] / 3.0) * T + a[2] / 2.0) * T + a[1]) * T + a[0] * logT + a[6]) +
           (-eos_R(t) * log(p / ORC_PSTD));
}
/* gpuThermo.H:287-299 */
static double th_Gstd(const thermo_t* t, double T, double logT) {
    const double* a = coeffs(t, T);
    return ((a[0] * (1.0 - logT) - (((a[4] / 20.0 * T + a[3] / 12.0) * T + a[2] / 6.0) * T + a[1] / 2.0) * T - a[6]) * T +
            a[5]);
}
/* gpuThermo.H:333-338 */
static double th_dCpdT_a(double T, const double* a) {
    return (((4.0 * a[4] * T + 3.0 * a[3]) * T + 2.0 * a[2]) * T + a[1]);
}
/* gpuThermo.H:80-87 */
static double th_K(const thermo_t* t, double T) {
    const double arg = -t->Y * th_Gstd(t, T, log(T)) / (ORC_RR * T);
    if (arg < 600) return exp(arg);
    return sqrt(ORC_VGREAT);
}
/* gpuThermo.H:106-113 */
static double th_Kc(const thermo_t* t, double T) {
    const double nm = t->Y / t->W;
    if (fabs(nm - ORC_SMALL) < ORC_VSMALL) return th_K(t, T);
    return th_K(t, T) * pow(ORC_PSTD / (ORC_RR * T), nm);
}
/* gpuThermo.H:139-169 */
static void th_KcAnddKcTbyKc(const thermo_t* t, double T, double* Kc_out, double* dK_out) {
    const double nm = t->Y / t->W;
    const double logT = log(T);
    const double Gstd = th_Gstd(t, T, logT);
    const int nm_is_small = fabs(nm - ORC_SMALL) < ORC_VSMALL;
    const double RRT = ORC_RR * T;
    double K;
    {
        const double arg = -t->Y * Gstd / RRT;
        K = arg < 600 ? exp(arg) : sqrt(ORC_VGREAT);
    }
    const double Kc = nm_is_small ? K : K * pow(ORC_PSTD / RRT, nm);
    const double S = th_S(t, ORC_PSTD, T, logT);
    double ret = (S + Gstd / T) * t->Y / RRT;
    if (!nm_is_small) ret = ret - nm / T;
    *Kc_out = Kc;
    *dK_out = ret;
}

/* -------------------------------------------------- loader arithmetic */

/* gpuPerfectGas.H:103-112 (operator+=) and gpuThermo.H:354-378 */
static void thermo_add(thermo_t* a, const thermo_t* b) {
    double Y1 = a->Y;
    const double sumY = a->Y + b->Y;
    if (fabs(sumY) > ORC_SMALL) a->W = sumY / (a->Y / a->W + b->Y / b->W);
    a->Y = sumY;
    if (fabs(a->Y) > ORC_SMALL) {
        Y1 /= a->Y;
        const double Y2 = b->Y / a->Y;
        a->Tlow = fmax(a->Tlow, b->Tlow);
        a->Thigh = fmin(a->Thigh, b->Thigh);
        for (int k = 0; k < 7; ++k) {
            a->high[k] = Y1 * a->high[k] + Y2 * b->high[k];
            a->low[k] = Y1 * a->low[k] + Y2 * b->low[k];
        }
    }
}

/* gpuPerfectGas.H:312-325 (operator==) and gpuThermo.H:442-470 */
static thermo_t thermo_eq(const thermo_t* t1, const thermo_t* t2) {
    thermo_t r;
    double diffY = t2->Y - t1->Y;
    if (fabs(diffY) < ORC_SMALL) diffY = ORC_SMALL;
    const double diffRW = t2->Y / t2->W - t1->Y / t1->W;
    double molWeight = ORC_GREAT;
    if (fabs(diffRW) > ORC_SMALL) molWeight = diffY / diffRW;
    r.Y = diffY;
    r.W = molWeight;
    const double Y1 = t2->Y / r.Y;
    const double Y2 = t1->Y / r.Y;
    for (int k = 0; k < 7; ++k) {
        r.high[k] = Y1 * t2->high[k] - Y2 * t1->high[k];
        r.low[k] = Y1 * t2->low[k] - Y2 * t1->low[k];
    }
    r.Tlow = fmax(t2->Tlow, t1->Tlow);
    r.Thigh = fmin(t2->Thigh, t1->Thigh);
    r.Tcommon = t2->Tcommon;
    return r;
}

/* (s * W) * thermo: gpuPerfectGas.H:300-302 and gpuThermo.H:428-436 */
static thermo_t thermo_scaled(const thermo_t* t, double stoich) {
    thermo_t r = *t;
    r.Y = (stoich * t->W) * t->Y;
    return r;
}

/* makeGpuReactions.H:18-59 — returns 0 on mass imbalance */
static int reaction_thermo(const mech_t* m, rxn_t* r) {
    thermo_t rhs = thermo_scaled(&m->th[r->rhs[0].index], r->rhs[0].stoich);
    for (int i = 1; i < r->nr; ++i) {
        thermo_t t = thermo_scaled(&m->th[r->rhs[i].index], r->rhs[i].stoich);
        thermo_add(&rhs, &t);
    }
    thermo_t lhs = thermo_scaled(&m->th[r->lhs[0].index], r->lhs[0].stoich);
    for (int i = 1; i < r->nl; ++i) {
        thermo_t t = thermo_scaled(&m->th[r->lhs[i].index], r->lhs[i].stoich);
        thermo_add(&lhs, &t);
    }
    if (fabs(lhs.Y - rhs.Y) > 0.1) return 0;
    r->th = thermo_eq(&lhs, &rhs);
    return 1;
}

/* gpuSpecieExponent.H:7-19 */
static int is_integer(double N) {
    const int X = (int)N;
    const double temp2 = N - X;
    return !(temp2 > 0);
}

static coeff_t make_coeff(int index, double stoich, double e) {
    coeff_t c;
    c.index = index;
    c.stoich = stoich;
    if (is_integer(e)) { /* makeGpuReactions.H:74-80 */
        c.is_int = 1;
        c.iexp = (int)e;
        c.sexp = (double)c.iexp;
    } else {
        c.is_int = 0;
        c.iexp = ORC_INT_MAX_10;
        c.sexp = e;
    }
    return c;
}

void* orc_mech_create(int nS, const double* W, const double* Tlow, const double* Thigh,
                      const double* Tcommon, const double* high_raw, const double* low_raw,
                      int nR, const int* rint, const double* rdbl, const double* eff,
                      double rxnTlow, double rxnThigh) {
    mech_t* m = (mech_t*)calloc(1, sizeof(mech_t));
    m->nS = nS;
    m->nR = nR;
    m->th = (thermo_t*)calloc((size_t)nS, sizeof(thermo_t));
    m->rx = (rxn_t*)calloc((size_t)(nR > 0 ? nR : 1), sizeof(rxn_t));
    m->eff = (double*)calloc((size_t)nR * nS + 1, sizeof(double));
    /* makeGpuThermo.H:41-44: coefficients x R = RR/W */
    for (int i = 0; i < nS; ++i) {
        thermo_t* t = &m->th[i];
        t->Y = 1.0;
        t->W = W[i];
        t->Tlow = Tlow[i];
        t->Thigh = Thigh[i];
        t->Tcommon = Tcommon[i];
        const double R = ORC_RR / W[i];
        for (int k = 0; k < 7; ++k) {
            t->high[k] = R * high_raw[7 * i + k];
            t->low[k] = R * low_raw[7 * i + k];
        }
    }
    for (int r = 0; r < nR; ++r) {
        const int* ri = rint + 24 * r;
        const double* rd = rdbl + 50 * r;
        rxn_t* x = &m->rx[r];
        x->type = ri[0];
        x->irr = ri[1];
        x->nl = ri[2];
        x->nr = ri[3];
        for (int i = 0; i < x->nl; ++i) x->lhs[i] = make_coeff(ri[4 + i], rd[i], rd[10 + i]);
        for (int i = 0; i < x->nr; ++i) x->rhs[i] = make_coeff(ri[14 + i], rd[20 + i], rd[30 + i]);
        x->A = rd[40];
        x->beta = rd[41];
        x->Ta = rd[42];
        x->Ainf = rd[43];
        x->betainf = rd[44];
        x->Tainf = rd[45];
        x->alpha = rd[46];
        x->Tsss = rd[47];
        x->Ts = rd[48];
        x->Tss = rd[49];
        x->Tlow = rxnTlow;
        x->Thigh = rxnThigh;
        if (x->type != 0) {
            memcpy(m->eff + (size_t)nS * r, eff + (size_t)nS * r, sizeof(double) * nS);
            x->eff = m->eff + (size_t)nS * r;
        } else {
            x->eff = NULL;
        }
        if (!reaction_thermo(m, x)) {
            orc_mech_destroy(m);
            return NULL;
        }
    }
    return m;
}

void orc_mech_destroy(void* h) {
    mech_t* m = (mech_t*)h;
    if (!m) return;
    free(m->th);
    free(m->rx);
    free(m->eff);
    free(m);
}

static void dump_thermo(const thermo_t* t, double* o) {
    o[0] = t->Y;
    o[1] = t->W;
    o[2] = t->Tlow;
    o[3] = t->Thigh;
    o[4] = t->Tcommon;
    for (int k = 0; k < 7; ++k) o[5 + k] = t->high[k];
    for (int k = 0; k < 7; ++k) o[12 + k] = t->low[k];
}

void orc_mech_tables(void* h, double* species_out, double* reaction_out, int* int_exp_out) {
    const mech_t* m = (const mech_t*)h;
    for (int i = 0; i < m->nS; ++i) dump_thermo(&m->th[i], species_out + 19 * i);
    for (int r = 0; r < m->nR; ++r) {
        const rxn_t* x = &m->rx[r];
        dump_thermo(&x->th, reaction_out + 19 * r);
        for (int i = 0; i < 10; ++i) {
            int_exp_out[20 * r + i] = i < x->nl ? x->lhs[i].is_int : -1;
            int_exp_out[20 * r + 10 + i] = i < x->nr ? x->rhs[i].is_int : -1;
        }
    }
}

void orc_thermo_eval(void* h, double p, double T, double* out) {
    const mech_t* m = (const mech_t*)h;
    for (int i = 0; i < m->nS; ++i) {
        const thermo_t* t = &m->th[i];
        double* o = out + 8 * i;
        const double* a = coeffs(t, T);
        o[0] = th_Cp_a(T, a);
        o[1] = th_Ha_a(T, a);
        o[2] = th_Ha_a(T, a) - th_Hf(t); /* Hs, gpuThermo.H:236-239 */
        o[3] = th_S(t, p, T, log(T));
        o[4] = th_Gstd(t, T, log(T));
        o[5] = th_dCpdT_a(T, a);
        o[6] = th_K(t, T);
        o[7] = th_Kc(t, T);
    }
}

/* ------------------------------------------------------------ reactions */

/* gpuSpecieExponent.H:21-36 */
static double integer_pow(double x, int e) {
    if (e == 0) return 1;
    double xx = e > 0 ? x : 1 / x;
    double y = 1;
    for (int i = e; i != 0; i /= 2) {
        if (i % 2) y *= xx;
        xx *= xx;
    }
    return y;
}
/* gpuSpecieExponent.H:103-110 */
static double specie_pow(double x, const coeff_t* c) {
    return c->is_int ? integer_pow(x, c->iexp) : pow(x, c->sexp);
}
/* speciePow(c, e - 1) with gpuSpecieExponent::operator- (gpuSpecieExponent.H:86-100) */
static double specie_pow_m1(double x, const coeff_t* c) {
    return c->is_int ? integer_pow(x, c->iexp - 1) : pow(x, c->sexp + (-1.0));
}

/* gpuArrheniusReactionRate.H:16-26 */
static double arrhenius(double A, double beta, double Ta, double T) {
    double ak = A;
    if (fabs(beta) > ORC_VSMALL) ak *= pow(T, beta);
    if (fabs(Ta) > ORC_VSMALL) ak *= exp(-Ta / T);
    return ak;
}
/* gpuThirdBodyEfficiencies.H:28-35 */
static double tb_M(const rxn_t* r, int nS, const double* c) {
    double M = 0;
    for (int i = 0; i < nS; ++i) M += r->eff[i] * c[i];
    return M;
}
/* gpuTroeFallOffFunction.H:27-47; gpuLindemannFallOffFunction.H:12-15 */
static double falloff_F(const rxn_t* r, double T, double Pr) {
    if (r->type == 2) return 1.0;
    const double logPr = log10(fmax(Pr, ORC_SMALL));
    const double Fcent = (1.0 - r->alpha) * exp(-T / r->Tsss) + r->alpha * exp(-T / r->Ts) + exp(-r->Tss / T);
    const double logFcent = log10(fmax(Fcent, ORC_SMALL));
    const double c = -0.4 - 0.67 * logFcent;
    const double d = 0.14;
    const double n = 0.75 - 1.27 * logFcent;
    const double x1 = n - d * (logPr + c);
    const double x2 = (logPr + c) / x1;
    const double x3 = 1.0 + x2 * x2;
    const double x4 = logFcent / x3;
    return pow(10.0, x4);
}

/* gpuReactionRate::operator() dispatch (gpuReactionRate.H:164-173) */
static double rate_k(const rxn_t* r, int nS, double T, const double* c) {
    switch (r->type) {
    case 0: return arrhenius(r->A, r->beta, r->Ta, T);
    case 1: /* gpuThirdBodyArrheniusReactionRate.H:39-44 */
        return tb_M(r, nS, c) * arrhenius(r->A, r->beta, r->Ta, T);
    default: { /* gpuFallOffReactionRate.H:39-51 */
        const double k0 = arrhenius(r->A, r->beta, r->Ta, T);
        const double kInf = arrhenius(r->Ainf, r->betainf, r->Tainf, T);
        const double M = tb_M(r, nS, c);
        const double Pr = k0 / kInf * M;
        const double F = falloff_F(r, T, Pr);
        return kInf * (Pr / (1.0 + Pr)) * F;
    }
    }
}

/* everything() (gpuArrheniusReactionRate.H:97-107, gpuThirdBodyArrheniusReactionRate.H:105-121,
 * gpuFallOffReactionRate.H:127-158); ddc written for types 1-3 */
static void rate_everything(const rxn_t* r, int nS, double T, const double* c, double* ddc,
                            double* k_out, double* dT_out) {
    if (r->type == 0) {
        const double Ak = arrhenius(r->A, r->beta, r->Ta, T);
        *k_out = Ak;
        *dT_out = Ak * (r->beta + r->Ta / T) / T;
    } else if (r->type == 1) {
        const double Ak = arrhenius(r->A, r->beta, r->Ta, T);
        const double dT = Ak * (r->beta + r->Ta / T) / T;
        for (int i = 0; i < nS; ++i) ddc[i] = r->eff[i] * Ak;
        const double M = tb_M(r, nS, c);
        *k_out = M * Ak;
        *dT_out = M * dT;
    } else {
        const double k0 = arrhenius(r->A, r->beta, r->Ta, T);
        const double kInf = arrhenius(r->Ainf, r->betainf, r->Tainf, T);
        const double M = tb_M(r, nS, c);
        const double Pr = k0 / kInf * M;
        const double F = falloff_F(r, T, Pr);
        const double temp = (Pr / (1.0 + Pr)) * F;
        const double k = kInf * temp;
        const double dkInfdT = arrhenius(r->Ainf, r->betainf, r->Tainf, T) * (r->betainf + r->Tainf / T) / T;
        const double ddT = dkInfdT * temp;
        for (int i = 0; i < nS; ++i) ddc[i] = 0.0;
        *k_out = k;
        *dT_out = ddT;
    }
}

/* gpuReaction.H:472-488 */
static double rxn_omega(const rxn_t* r, int nS, double p, double T, const double* c) {
    (void)p;
    const double clippedT = fmin(fmax(T, r->Tlow), r->Thigh);
    const double kf = rate_k(r, nS, clippedT, c);
    const double kr = r->irr ? 0.0 : kf / th_Kc(&r->th, clippedT);
    double Cf = 1.0, Cr = 1.0;
    for (int i = 0; i < r->nl; ++i) Cf *= specie_pow(c[r->lhs[i].index], &r->lhs[i]);
    for (int i = 0; i < r->nr; ++i) Cr *= specie_pow(c[r->rhs[i].index], &r->rhs[i]);
    return kf * Cf - kr * Cr;
}

typedef struct {
    double omega, dwdT, kf, kr;
    double dCf[ORC_MAXW], dCr[ORC_MAXW];
} params_t;

/* computeReactionParameters, gpuReaction.H:650-702 (with calcdCfdcj/calcdCrdcj
 * :388-470) */
static params_t rxn_params(const rxn_t* r, int nS, const double* c, double T, double* ddc) {
    params_t ret;
    memset(&ret, 0, sizeof(ret));
    double kf, ddT;
    rate_everything(r, nS, T, c, ddc, &kf, &ddT);
    double lhsPow[ORC_MAXW];
    for (int i = 0; i < r->nl; ++i) lhsPow[i] = specie_pow(c[r->lhs[i].index], &r->lhs[i]);
    double Cf = 1.0;
    for (int i = 0; i < r->nl; ++i) Cf *= lhsPow[i];
    for (int j = 0; j < r->nl; ++j) {
        double d = 1;
        for (int i = 0; i < r->nl; ++i) {
            if (i == j) {
                d *= r->lhs[i].sexp * specie_pow_m1(c[r->lhs[i].index], &r->lhs[i]);
            } else {
                d *= lhsPow[i];
            }
        }
        ret.dCf[j] = d;
    }
    ret.dwdT = Cf * ddT;
    ret.omega = Cf * kf;
    for (int j = 0; j < ORC_MAXW; ++j) ret.dCf[j] *= kf;
    double Cr = 0.0, Kc = 1.0;
    ret.kf = kf;
    ret.kr = 0.0;
    if (!r->irr) {
        double dKcdTbyV;
        th_KcAnddKcTbyKc(&r->th, T, &Kc, &dKcdTbyV);
        const double kr = kf / Kc;
        double rhsPow[ORC_MAXW];
        for (int i = 0; i < r->nr; ++i) rhsPow[i] = specie_pow(c[r->rhs[i].index], &r->rhs[i]);
        Cr = 1.0;
        for (int i = 0; i < r->nr; ++i) Cr *= rhsPow[i];
        const double dkrdT = ddT / Kc - kr * dKcdTbyV;
        ret.dwdT -= Cr * dkrdT;
        ret.omega -= Cr * kr;
        for (int j = 0; j < r->nr; ++j) {
            double d = 1;
            for (int i = 0; i < r->nr; ++i) {
                if (i == j) {
                    d *= r->rhs[i].sexp * specie_pow_m1(c[r->rhs[i].index], &r->rhs[i]);
                } else {
                    d *= rhsPow[i];
                }
            }
            ret.dCr[j] = d;
        }
        for (int j = 0; j < ORC_MAXW; ++j) ret.dCr[j] *= kr;
        ret.kr = kr;
    }
    if (r->type != 0) {
        const double temp = (Cf - Cr / Kc);
        for (int j = 0; j < nS; ++j) ddc[j] *= temp;
    }
    return ret;
}

void orc_reaction_eval(void* h, const double* y, double* out) {
    const mech_t* m = (const mech_t*)h;
    const int nS = m->nS;
    double* c = (double*)malloc(sizeof(double) * (size_t)nS);
    double* ddc = (double*)malloc(sizeof(double) * (size_t)nS);
    const double T = y[nS], p = y[nS + 1];
    double rhoM = 0.0;
    for (int i = 0; i < nS; ++i) {
        const double yi = fmax(y[i], 0.0);
        rhoM += yi / eos_rho(&m->th[i], p, T);
        c[i] = yi / m->th[i].W;
    }
    rhoM = 1.0 / rhoM;
    for (int i = 0; i < nS; ++i) c[i] *= rhoM;
    for (int r = 0; r < m->nR; ++r) {
        const rxn_t* x = &m->rx[r];
        double* o = out + 6 * r;
        o[0] = rate_k(x, nS, T, c);
        o[1] = x->irr ? 0.0 : rate_k(x, nS, T, c) / th_Kc(&x->th, T);
        o[2] = rxn_omega(x, nS, p, T, c);
        th_KcAnddKcTbyKc(&x->th, T, &o[3], &o[4]);
        const params_t prm = rxn_params(x, nS, c, T, ddc);
        o[5] = prm.dwdT;
    }
    free(c);
    free(ddc);
}

/* ----------------------------------------------------------- ODE system */

typedef struct {
    int nS, n;
    double *c, *Cp, *Ha, *ddc, *temp;
    double *dydx0, *yTemp, *dydx, *dfdx, *k1, *k2, *k3, *k4, *err, *vv, *J;
    int* piv;
} ws_t;

static void ws_init(ws_t* w, int nS) {
    const int n = nS + 2;
    w->nS = nS;
    w->n = n;
    w->c = (double*)calloc((size_t)n, sizeof(double));
    w->Cp = (double*)calloc((size_t)n, sizeof(double));
    w->Ha = (double*)calloc((size_t)n, sizeof(double));
    w->ddc = (double*)calloc((size_t)n, sizeof(double));
    w->temp = (double*)calloc((size_t)n, sizeof(double));
    w->dydx0 = (double*)calloc((size_t)n, sizeof(double));
    w->yTemp = (double*)calloc((size_t)n, sizeof(double));
    w->dydx = (double*)calloc((size_t)n, sizeof(double));
    w->dfdx = (double*)calloc((size_t)n, sizeof(double));
    w->k1 = (double*)calloc((size_t)n, sizeof(double));
    w->k2 = (double*)calloc((size_t)n, sizeof(double));
    w->k3 = (double*)calloc((size_t)n, sizeof(double));
    w->k4 = (double*)calloc((size_t)n, sizeof(double));
    w->err = (double*)calloc((size_t)n, sizeof(double));
    w->vv = (double*)calloc((size_t)n, sizeof(double));
    w->J = (double*)calloc((size_t)n * n, sizeof(double));
    w->piv = (int*)calloc((size_t)n, sizeof(int));
}

static void ws_free(ws_t* w) {
    free(w->c); free(w->Cp); free(w->Ha); free(w->ddc); free(w->temp);
    free(w->dydx0); free(w->yTemp); free(w->dydx); free(w->dfdx);
    free(w->k1); free(w->k2); free(w->k3); free(w->k4); free(w->err);
    free(w->vv); free(w->J); free(w->piv);
}

/* gpuODESystem.H:164-196 with gpuMixture::computeDerivativeRequired
 * (gpuMixture.H:88-121), dYdT (:40-48) and dTdt (:53-63) */
static void derivatives(const mech_t* m, ws_t* w, const double* y, double* dydx) {
    const int nS = m->nS, n = nS + 2;
    for (int i = 0; i < n; ++i) dydx[i] = 0;
    const double T = y[nS], p = y[nS + 1];
    double rhoM = 0.0, CpM = 0.0;
    for (int i = 0; i < nS; ++i) {
        const double yi = fmax(y[i], 0.0);
        const thermo_t* t = &m->th[i];
        const double rhoi = eos_rho(t, p, T);
        const double* a = coeffs(t, T);
        const double Cpi = th_Cp_a(T, a);
        const double Hai = th_Ha_a(T, a);
        rhoM += yi / rhoi;
        CpM += yi * Cpi;
        w->Ha[i] = Hai;
        w->c[i] = yi / t->W;
    }
    rhoM = 1.0 / rhoM;
    for (int i = 0; i < nS; ++i) w->c[i] *= rhoM;
    for (int r = 0; r < m->nR; ++r) {
        const rxn_t* x = &m->rx[r];
        const double omega = rxn_omega(x, nS, p, T, w->c);
        for (int i = 0; i < x->nl; ++i) dydx[x->lhs[i].index] -= x->lhs[i].stoich * omega;
        for (int i = 0; i < x->nr; ++i) dydx[x->rhs[i].index] += x->rhs[i].stoich * omega;
    }
    for (int i = 0; i < nS; ++i) dydx[i] *= m->th[i].W / rhoM;
    double ret = 0.0;
    for (int i = 0; i < nS; ++i) ret -= dydx[i] * w->Ha[i];
    dydx[nS] = ret / CpM;
    dydx[nS + 1] = 0.0;
}

#define JIJ(i, j) J[(size_t)(i) * n + (j)]

/* gpuODESystem.H:198-281 with computeJacobianRequired (gpuMixture.H:33-77),
 * the per-reaction contributions (gpuReaction.H:547-648) and ddY_dcdY,
 * ddT_dtdY, ddT_dtdT (gpuODESystem.H:65-146) */
static void jacobian(const mech_t* m, ws_t* w, const double* y, double* dfdx, double* J) {
    const int nS = m->nS, n = nS + 2;
    for (int i = 0; i < n; ++i) dfdx[i] = 0.0;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) JIJ(i, j) = 0.0;
    const double T = y[nS], p = y[nS + 1];
    double rhoM = 0.0, CpM = 0.0, dCpMdT = 0.0, alphav = 0.0;
    for (int i = 0; i < nS; ++i) {
        const double yi = fmax(y[i], 0.0);
        const thermo_t* t = &m->th[i];
        const double rhoi = eos_rho(t, p, T);
        const double vi = 1.0 / rhoi;
        const double* a = coeffs(t, T);
        const double Cpi = th_Cp_a(T, a);
        const double Hai = th_Ha_a(T, a);
        const double dCpMdTi = th_dCpdT_a(T, a);
        rhoM += yi / rhoi;
        CpM += yi * Cpi;
        dCpMdT += yi * dCpMdTi;
        alphav += yi * vi * (1.0 / T);
        w->Cp[i] = Cpi;
        w->Ha[i] = Hai;
        w->c[i] = yi / t->W;
    }
    rhoM = 1.0 / rhoM;
    alphav = alphav * rhoM;
    for (int i = 0; i < nS; ++i) w->c[i] *= rhoM;
    const double* c = w->c;
    double* ddc = w->ddc;
    for (int ri = 0; ri < m->nR; ++ri) {
        const rxn_t* x = &m->rx[ri];
        const params_t prm = rxn_params(x, nS, c, T, ddc);
        /* dNdtByV(params, dfdx) */
        for (int i = 0; i < x->nl; ++i) dfdx[x->lhs[i].index] -= x->lhs[i].stoich * prm.omega;
        for (int i = 0; i < x->nr; ++i) dfdx[x->rhs[i].index] += x->rhs[i].stoich * prm.omega;
        /* jac_dCfdcj_contribution */
        for (int j = 0; j < x->nl; ++j) {
            const int sj = x->lhs[j].index;
            for (int i = 0; i < x->nl; ++i) JIJ(x->lhs[i].index, sj) -= x->lhs[i].stoich * prm.dCf[j];
            for (int i = 0; i < x->nr; ++i) JIJ(x->rhs[i].index, sj) += x->rhs[i].stoich * prm.dCf[j];
        }
        /* jac_dCrdcj_contribution */
        for (int j = 0; j < x->nr; ++j) {
            const int sj = x->rhs[j].index;
            for (int i = 0; i < x->nl; ++i) JIJ(x->lhs[i].index, sj) += x->lhs[i].stoich * prm.dCr[j];
            for (int i = 0; i < x->nr; ++i) JIJ(x->rhs[i].index, sj) -= x->rhs[i].stoich * prm.dCr[j];
        }
        /* jac_dCdT_contribution */
        for (int i = 0; i < x->nl; ++i) JIJ(x->lhs[i].index, nS) -= x->lhs[i].stoich * prm.dwdT;
        for (int i = 0; i < x->nr; ++i) JIJ(x->rhs[i].index, nS) += x->rhs[i].stoich * prm.dwdT;
        /* jac_dCdC_contribution */
        if (x->type != 0) {
            for (int i = 0; i < x->nl; ++i) {
                double* row = &JIJ(x->lhs[i].index, 0);
                for (int j = 0; j < nS; ++j) row[j] -= x->lhs[i].stoich * ddc[j];
            }
            for (int i = 0; i < x->nr; ++i) {
                double* row = &JIJ(x->rhs[i].index, 0);
                for (int j = 0; j < nS; ++j) row[j] += x->rhs[i].stoich * ddc[j];
            }
        }
    }
    for (int i = 0; i < nS; ++i) dfdx[i] *= m->th[i].W / rhoM;
    {
        double ret = 0.0;
        for (int i = 0; i < nS; ++i) ret -= dfdx[i] * w->Ha[i];
        dfdx[nS] = ret / CpM;
    }
    dfdx[nS + 1] = 0.0;
    /* ddY_dcdY */
    double* temp = w->temp;
    for (int i = 0; i < nS; ++i) {
        const double WiByrhoM = m->th[i].W / rhoM;
        for (int j = 0; j < nS + 2; ++j) temp[j] = JIJ(i, j);
        for (int j = 0; j < nS; ++j) {
            const double rhoMByWi = rhoM / m->th[j].W;
            const double vj = 1.0 / eos_rho(&m->th[j], p, T);
            JIJ(i, j) = WiByrhoM * temp[j] * rhoMByWi + rhoM * vj * dfdx[i];
        }
        double ddNidtByVdT = temp[nS];
        for (int j = 0; j < nS; ++j) ddNidtByVdT -= temp[j] * c[j] * alphav;
        JIJ(i, nS) = WiByrhoM * ddNidtByVdT + alphav * dfdx[i];
        JIJ(i, nS + 1) = 0.0;
    }
    /* ddT_dtdY */
    for (int i = 0; i < nS; ++i) {
        JIJ(nS, i) = 0.0;
        for (int j = 0; j < nS; ++j) JIJ(nS, i) -= JIJ(j, i) * w->Ha[j];
        const double Cpi = w->Cp[i];
        JIJ(nS, i) -= Cpi * dfdx[nS];
        JIJ(nS, i) /= CpM;
    }
    /* ddT_dtdT */
    JIJ(nS, nS) = 0.0;
    for (int i = 0; i < nS; ++i) JIJ(nS, nS) -= dfdx[i] * w->Cp[i] + JIJ(i, nS) * w->Ha[i];
    JIJ(nS, nS) -= dfdx[nS] * dCpMdT;
    JIJ(nS, nS) /= CpM;
}

void orc_derivatives(void* h, int nst, const double* y, double* dydx) {
    const mech_t* m = (const mech_t*)h;
    ws_t w;
    ws_init(&w, m->nS);
    for (int s = 0; s < nst; ++s) derivatives(m, &w, y + (size_t)(m->nS + 2) * s, dydx + (size_t)(m->nS + 2) * s);
    ws_free(&w);
}

void orc_jacobian(void* h, int nst, const double* y, double* dfdx, double* J) {
    const mech_t* m = (const mech_t*)h;
    const int n = m->nS + 2;
    ws_t w;
    ws_init(&w, m->nS);
    for (int s = 0; s < nst; ++s) jacobian(m, &w, y + (size_t)n * s, dfdx + (size_t)n * s, J + (size_t)n * n * s);
    ws_free(&w);
}

/* --------------------------------------------------------------- LU */

/* ludecompose.H:9-92 */
static void lu_decompose(int m, double* A, int* piv, double* vv) {
    for (int i = 0; i < m; i++) {
        double largest = 0.0, temp;
        const double* Ai = A + (size_t)i * m;
        for (int j = 0; j < m; j++) {
            if ((temp = fabs(Ai[j])) > largest) largest = temp;
        }
        vv[i] = 1.0 / largest;
    }
    for (int j = 0; j < m; j++) {
        double* Aj = A + (size_t)j * m;
        for (int i = 0; i < j; i++) {
            double* Ai = A + (size_t)i * m;
            double sum = Ai[j];
            for (int k = 0; k < i; k++) sum -= Ai[k] * A[(size_t)k * m + j];
            Ai[j] = sum;
        }
        int iMax = 0;
        double largest = 0.0;
        for (int i = j; i < m; i++) {
            double* Ai = A + (size_t)i * m;
            double sum = Ai[j];
            for (int k = 0; k < j; k++) sum -= Ai[k] * A[(size_t)k * m + j];
            Ai[j] = sum;
            double temp;
            if ((temp = vv[i] * fabs(sum)) >= largest) {
                largest = temp;
                iMax = i;
            }
        }
        piv[j] = iMax;
        if (j != iMax) {
            double* Am = A + (size_t)iMax * m;
            for (int k = 0; k < m; k++) {
                const double t = Aj[k];
                Aj[k] = Am[k];
                Am[k] = t;
            }
            vv[iMax] = vv[j];
        }
        if (Aj[j] == 0.0) Aj[j] = ORC_SMALL;
        if (j != m - 1) {
            const double rDiag = 1.0 / Aj[j];
            for (int i = j + 1; i < m; i++) A[(size_t)i * m + j] *= rDiag;
        }
    }
}

/* ludecompose.H:94-130 */
static void lu_backsubstitute(int m, const double* LU, const int* piv, double* b) {
    int ii = 0;
    for (int i = 0; i < m; i++) {
        const int ip = piv[i];
        double sum = b[ip];
        b[ip] = b[i];
        const double* Li = LU + (size_t)i * m;
        if (ii != 0) {
            for (int j = ii - 1; j < i; j++) sum -= Li[j] * b[j];
        } else if (sum != 0.0) {
            ii = i + 1;
        }
        b[i] = sum;
    }
    for (int i = m - 1; i >= 0; i--) {
        double sum = b[i];
        const double* Li = LU + (size_t)i * m;
        for (int j = i + 1; j < m; j++) sum -= Li[j] * b[j];
        b[i] = sum / Li[i];
    }
}

void orc_lu(int m, int n_mats, double* A, int* piv, double* b) {
    double* vv = (double*)malloc(sizeof(double) * (size_t)m);
    for (int k = 0; k < n_mats; ++k) {
        lu_decompose(m, A + (size_t)m * m * k, piv + (size_t)m * k, vv);
        lu_backsubstitute(m, A + (size_t)m * m * k, piv + (size_t)m * k, b + (size_t)m * k);
    }
    free(vv);
}

/* -------------------------------------------------------- Rosenbrock */

/* gpuAdaptiveSolver.H:51-73 */
static void decomposed_jacobian(const mech_t* m, ws_t* w, double dx, double gamma, const double* y0) {
    const int n = m->nS + 2;
    double* J = w->J;
    jacobian(m, w, y0, w->dfdx, J);
    const double temp = 1.0 / (gamma * dx);
    for (int i = 0; i < n; i++) {
        for (int j = 0; j < n; j++) JIJ(i, j) = -JIJ(i, j);
        JIJ(i, i) += temp;
    }
    lu_decompose(n, J, w->piv, w->vv);
}

/* normaliseError.H:6-29 */
static double normalise_error(int n, const double* y0, const double* y, const double* err, double absTol,
                              double relTol) {
    double maxErr = 0.0;
    for (int i = 0; i < n; ++i) {
        const double tol = absTol + relTol * fmax(fabs(y0[i]), fabs(y[i]));
        const double t = fabs(err[i]) / tol;
        maxErr = fmax(maxErr, t);
    }
    return maxErr;
}

/* gpuRosenbrock12.H:14-31, 53-103 */
static double ros12(const mech_t* m, ws_t* w, const orc_ode_inputs* o, const double* y0, const double* dydx0,
                    double dx, double* y) {
    const double gamma = 1.0 + 1.0 / 1.414213562373095;
    const double a21 = 1.0 / gamma, c21 = -2.0 / gamma;
    const double b1 = (3.0 / 2.0) / gamma, b2 = (1.0 / 2.0) / gamma;
    const double e1 = b1 - 1.0 / gamma, e2 = b2;
    const double d1 = gamma, d2 = -gamma;
    const int n = m->nS + 2;
    decomposed_jacobian(m, w, dx, gamma, y0);
    for (int i = 0; i < n; ++i) w->k1[i] = dydx0[i] + dx * d1 * w->dfdx[i];
    lu_backsubstitute(n, w->J, w->piv, w->k1);
    for (int i = 0; i < n; ++i) y[i] = y0[i] + a21 * w->k1[i];
    derivatives(m, w, y, w->dydx);
    for (int i = 0; i < n; ++i) w->k2[i] = w->dydx[i] + dx * d2 * w->dfdx[i] + c21 * w->k1[i] / dx;
    lu_backsubstitute(n, w->J, w->piv, w->k2);
    for (int i = 0; i < n; ++i) {
        y[i] = y0[i] + b1 * w->k1[i] + b2 * w->k2[i];
        w->err[i] = e1 * w->k1[i] + e2 * w->k2[i];
    }
    return normalise_error(n, y0, y, w->err, o->absTol, o->relTol);
}

/* gpuRosenbrock23.H:13-37, 58-116 */
static double ros23(const mech_t* m, ws_t* w, const orc_ode_inputs* o, const double* y0, const double* dydx0,
                    double dx, double* y) {
    const double a21 = 1;
    const double c21 = -1.0156171083877702091975600115545;
    const double c31 = 4.0759956452537699824805835358067;
    const double c32 = 9.2076794298330791242156818474003;
    const double b1 = 1, b2 = 6.1697947043828245592553615689730, b3 = -0.4277225654321857332623837380651;
    const double e1 = 0.5, e2 = -2.9079558716805469821718236208017, e3 = 0.2235406989781156962736090927619;
    const double gamma = 0.43586652150845899941601945119356;
    const double d1 = 0.43586652150845899941601945119356;
    const double d2 = 0.24291996454816804366592249683314;
    const double d3 = 2.1851380027664058511513169485832;
    const int n = m->nS + 2;
    decomposed_jacobian(m, w, dx, gamma, y0);
    for (int i = 0; i < n; ++i) w->k1[i] = dydx0[i] + dx * d1 * w->dfdx[i];
    lu_backsubstitute(n, w->J, w->piv, w->k1);
    for (int i = 0; i < n; ++i) y[i] = y0[i] + a21 * w->k1[i];
    derivatives(m, w, y, w->dydx);
    for (int i = 0; i < n; ++i) w->k2[i] = w->dydx[i] + dx * d2 * w->dfdx[i] + c21 * w->k1[i] / dx;
    lu_backsubstitute(n, w->J, w->piv, w->k2);
    for (int i = 0; i < n; ++i) w->k3[i] = w->dydx[i] + dx * d3 * w->dfdx[i] + (c31 * w->k1[i] + c32 * w->k2[i]) / dx;
    lu_backsubstitute(n, w->J, w->piv, w->k3);
    for (int i = 0; i < n; ++i) {
        y[i] = y0[i] + b1 * w->k1[i] + b2 * w->k2[i] + b3 * w->k3[i];
        w->err[i] = e1 * w->k1[i] + e2 * w->k2[i] + e3 * w->k3[i];
    }
    return normalise_error(n, y0, y, w->err, o->absTol, o->relTol);
}

/* gpuRosenbrock34.H:13-46, 67-139 */
static double ros34(const mech_t* m, ws_t* w, const orc_ode_inputs* o, const double* y0, const double* dydx0,
                    double dx, double* y) {
    const double a21 = 2.0, a31 = 48.0 / 25.0, a32 = 6.0 / 25.0;
    const double c21 = -8.0, c31 = 372.0 / 25.0, c32 = 12.0 / 5.0;
    const double c41 = -112.0 / 125.0, c42 = -54.0 / 125.0, c43 = -2.0 / 5.0;
    const double b1 = 19.0 / 9.0, b2 = 1.0 / 2.0, b3 = 25.0 / 108.0, b4 = 125.0 / 108.0;
    const double e1 = 34.0 / 108.0, e2 = 7.0 / 36.0, e4 = 125.0 / 108.0;
    const double gamma = 1.0 / 2.0;
    const double d1 = 1.0 / 2.0, d2 = -3.0 / 2.0, d3 = 605.0 / 250.0, d4 = 29.0 / 250.0;
    const int n = m->nS + 2;
    decomposed_jacobian(m, w, dx, gamma, y0);
    for (int i = 0; i < n; ++i) w->k1[i] = dydx0[i] + dx * d1 * w->dfdx[i];
    lu_backsubstitute(n, w->J, w->piv, w->k1);
    for (int i = 0; i < n; ++i) y[i] = y0[i] + a21 * w->k1[i];
    derivatives(m, w, y, w->dydx);
    for (int i = 0; i < n; ++i) w->k2[i] = w->dydx[i] + dx * d2 * w->dfdx[i] + c21 * w->k1[i] / dx;
    lu_backsubstitute(n, w->J, w->piv, w->k2);
    for (int i = 0; i < n; ++i) y[i] = y0[i] + a31 * w->k1[i] + a32 * w->k2[i];
    derivatives(m, w, y, w->dydx);
    for (int i = 0; i < n; ++i) w->k3[i] = w->dydx[i] + dx * d3 * w->dfdx[i] + (c31 * w->k1[i] + c32 * w->k2[i]) / dx;
    lu_backsubstitute(n, w->J, w->piv, w->k3);
    for (int i = 0; i < n; ++i)
        w->k4[i] = w->dydx[i] + dx * d4 * w->dfdx[i] + (c41 * w->k1[i] + c42 * w->k2[i] + c43 * w->k3[i]) / dx;
    lu_backsubstitute(n, w->J, w->piv, w->k4);
    for (int i = 0; i < n; ++i) {
        y[i] = y0[i] + b1 * w->k1[i] + b2 * w->k2[i] + b3 * w->k3[i] + b4 * w->k4[i];
        w->err[i] = e1 * w->k1[i] + e2 * w->k2[i] + e4 * w->k4[i];
    }
    return normalise_error(n, y0, y, w->err, o->absTol, o->relTol);
}

static double attempt(const mech_t* m, ws_t* w, const orc_ode_inputs* o, const double* y0, const double* dydx0,
                      double dx, double* y) {
    if (o->solver == 12) return ros12(m, w, o, y0, dydx0, dx, y);
    if (o->solver == 23) return ros23(m, w, o, y0, dydx0, dx, y);
    return ros34(m, w, o, y0, dydx0, dx, y);
}

void orc_attempt(void* h, const orc_ode_inputs* o, int nst, const double* y0, const double* dydx0,
                 const double* dx, double* y, double* err) {
    const mech_t* m = (const mech_t*)h;
    const int n = m->nS + 2;
    ws_t w;
    ws_init(&w, m->nS);
    for (int s = 0; s < nst; ++s)
        err[s] = attempt(m, &w, o, y0 + (size_t)n * s, dydx0 + (size_t)n * s, dx[s], y + (size_t)n * s);
    ws_free(&w);
}

/* The frozen-step replay of a recorded integration (the map the adjoint
 * differentiates): y_{k+1} = attempt(y_k, f(y_k), h_k) for k < n_steps, each
 * step adaptiveSolve's derivatives call (gpuAdaptiveSolver.H:96) and one
 * attempt with the recorded size, then singleCellSolver's max(0, Y)
 * (singleCellSolver.H:41-45). y [nS + 2] in place. */
void orc_replay(void* h, const orc_ode_inputs* o, int n_steps, const double* steps, double* y) {
    const mech_t* m = (const mech_t*)h;
    const int n = m->nS + 2;
    ws_t w;
    ws_init(&w, m->nS);
    for (int k = 0; k < n_steps; ++k) {
        derivatives(m, &w, y, w.dydx0);
        attempt(m, &w, o, y, w.dydx0, steps[k], w.yTemp);
        for (int i = 0; i < n; ++i) y[i] = w.yTemp[i];
    }
    for (int i = 0; i < m->nS; ++i) y[i] = fmax(0.0, y[i]);
    ws_free(&w);
}

/* adaptiveSolve, gpuAdaptiveSolver.H:83-134. Returns 0, or CELL_STEP_UNDERFLOW
 * where the reference prints and asserts (:111-114). */
static int adaptive_solve(const mech_t* m, ws_t* w, const orc_ode_inputs* o, double* x, double* y, double* dxTry,
                          long* attempts) {
    const int n = m->nS + 2;
    double dx = *dxTry;
    double err = 0.0;
    derivatives(m, w, y, w->dydx0);
    do {
        err = attempt(m, w, o, y, w->dydx0, dx, w->yTemp);
        ++*attempts;
        if (err > 1) {
            const double scale = fmax(o->safeScale * pow(err, -o->alphaDec), o->minScale);
            dx *= scale;
            if (dx < ORC_VSMALL) return CELL_STEP_UNDERFLOW;
        }
    } while (err > 1.0);
    *x += dx;
    for (int i = 0; i < n; ++i) y[i] = w->yTemp[i];
    if (err > pow(o->maxScale / o->safeScale, -1.0 / o->alphaInc)) {
        *dxTry = fmin(fmax(o->safeScale * pow(err, -o->alphaInc), o->minScale), o->maxScale) * dx;
    } else {
        *dxTry = o->safeScale * o->maxScale * dx;
    }
    return 0;
}

/* odeSolve, gpuODESolverBase.H:67-111 with stepState (stepState.H:8-26) */
static int ode_solve(const mech_t* m, ws_t* w, const orc_ode_inputs* o, double xStart, double xEnd, double* y,
                     double* dxTry, long* accepted, long* attempts) {
    double step_dxTry = *dxTry;
    int last = 0;
    double x = xStart;
    for (int nStep = 0; nStep < o->maxSteps; nStep++) {
        const double dxTry0 = step_dxTry;
        if ((x + step_dxTry - xEnd) * (x + step_dxTry - xStart) > 0) {
            last = 1;
            step_dxTry = xEnd - x;
        }
        const int st = adaptive_solve(m, w, o, &x, y, &step_dxTry, attempts);
        if (st) return st;
        ++*accepted;
        if ((x - xEnd) * (xEnd - xStart) >= 0) {
            if (nStep > 0 && last) step_dxTry = dxTry0;
            *dxTry = step_dxTry;
            return CELL_OK;
        }
    }
    return CELL_MAX_STEPS;
}

/* singleCellSolver::operator(), singleCellSolver.H:27-51, with per-cell status
 * and counters (accepted, attempts). */
void orc_cells(void* h, const orc_ode_inputs* o, double Treact, int nc, double deltaT, const double* deltaT_cell,
               double* Y, double* deltaTChem, int* counts, int* status, int nthreads) {
    const mech_t* m = (const mech_t*)h;
    const int nS = m->nS, n = nS + 2;
#ifdef _OPENMP
#pragma omp parallel num_threads(nthreads > 0 ? nthreads : omp_get_max_threads())
#endif
    {
        ws_t w;
        ws_init(&w, nS);
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 1)
#endif
        for (int c = 0; c < nc; ++c) {
            double* y = Y + (size_t)n * c;
            const double dT = deltaT_cell ? deltaT_cell[c] : deltaT;
            long acc = 0, att = 0;
            int st = CELL_OK;
            if (y[nS] > Treact) {
                double timeLeft = dT;
                while (timeLeft > ORC_SMALL) {
                    const double dt = timeLeft;
                    const int s = ode_solve(m, &w, o, 0, dt, y, &deltaTChem[c], &acc, &att);
                    if (s != CELL_OK && st == CELL_OK) st = s;
                    if (s == CELL_STEP_UNDERFLOW) break;
                    for (int i = 0; i < n; ++i) {
                        if (!isfinite(y[i]) && st == CELL_OK) st = CELL_NONFINITE;
                    }
                    for (int i = 0; i < nS; i++) y[i] = fmax(0.0, y[i]);
                    timeLeft -= dt;
                }
            } else {
                deltaTChem[c] = dT;
                st = CELL_SKIPPED;
            }
            if (counts) {
                counts[2 * c] = (int)acc;
                counts[2 * c + 1] = (int)att;
            }
            if (status) status[c] = st;
        }
        ws_free(&w);
    }
    (void)nthreads;
}

/* gpuKernelEvaluator.cu:84-96 */
double orc_compute_rr_host(int nc, int nS, double deltaT, double deltaTChemMax, const double* rho, const double* Y0,
                           const double* Ynew, double* deltaTChemNew, double* RR) {
    const int n = nS + 2;
    for (int j = 0; j < nc; ++j)
        for (int i = 0; i < nS; ++i)
            RR[(size_t)j * nS + i] = rho[j] * (Ynew[(size_t)j * n + i] - Y0[(size_t)j * n + i]) / deltaT;
    double mn = deltaTChemNew[0];
    for (int j = 1; j < nc; ++j) mn = fmin(mn, deltaTChemNew[j]);
    for (int j = 0; j < nc; ++j) deltaTChemNew[j] = fmin(deltaTChemNew[j], deltaTChemMax);
    return mn;
}

/* ---- the plugin's per-cell side paths (gpuChemistryModel.C), on the
 * concentrations c_i = rho Y_i / W_i of the thermo's density ---- */

static void field_c(const mech_t* m, double rho, const double* y, double* c) {
    for (int i = 0; i < m->nS; ++i) c[i] = rho * y[i] / m->th[i].W; /* :163-166 */
}

/* calculate() :145-186 (RR [n][nS]) and tc() :366-427 ([n]); either may be NULL */
void orc_cell_fields(void* h, int nc, const double* rho, const double* y, double* RR, double* tc) {
    const mech_t* m = (const mech_t*)h;
    const int nS = m->nS, ne = nS + 2;
    double* c = (double*)malloc(sizeof(double) * (nS > 0 ? nS : 1));
    double* dN = (double*)malloc(sizeof(double) * (nS > 0 ? nS : 1));
    for (int j = 0; j < nc; ++j) {
        const double* yj = y + (size_t)j * ne;
        const double T = yj[nS], p = yj[nS + 1];
        field_c(m, rho[j], yj, c);
        if (RR) {
            for (int i = 0; i < nS; ++i) dN[i] = 0.0;
            for (int r = 0; r < m->nR; ++r) { /* gpuReaction.H:490-508 */
                const rxn_t* R = &m->rx[r];
                const double om = rxn_omega(R, nS, p, T, c);
                for (int k = 0; k < R->nl; ++k) dN[R->lhs[k].index] -= R->lhs[k].stoich * om;
                for (int k = 0; k < R->nr; ++k) dN[R->rhs[k].index] += R->rhs[k].stoich * om;
            }
            for (int i = 0; i < nS; ++i) RR[(size_t)j * nS + i] = dN[i] * m->th[i].W;
        }
        if (tc) {
            double sumW = 0, sumWRateByCTot = 0;
            for (int r = 0; r < m->nR; ++r) {
                const rxn_t* R = &m->rx[r];
                const double clippedT = fmin(fmax(T, R->Tlow), R->Thigh);
                const double kf = rate_k(R, nS, clippedT, c);
                const double kr = R->irr ? 0.0 : kf / th_Kc(&R->th, clippedT);
                double Cf = 1.0, Cr = 1.0;
                for (int k = 0; k < R->nl; ++k) Cf *= specie_pow(c[R->lhs[k].index], &R->lhs[k]);
                for (int k = 0; k < R->nr; ++k) Cr *= specie_pow(c[R->rhs[k].index], &R->rhs[k]);
                const double omegaf = kf * Cf, omegar = kr * Cr;
                double wf = 0;
                for (int k = 0; k < R->nr; ++k) wf += R->rhs[k].stoich * omegaf;
                sumW += wf;
                sumWRateByCTot += wf * wf;
                double wr = 0;
                for (int k = 0; k < R->nl; ++k) wr += R->lhs[k].stoich * omegar;
                sumW += wr;
                sumWRateByCTot += wr * wr;
            }
            double ctot = 0;
            for (int i = 0; i < nS; ++i) ctot += c[i];
            tc[j] = sumWRateByCTot == 0 ? ORC_VGREAT : sumW / sumWRateByCTot * ctot;
        }
    }
    free(c);
    free(dN);
}

/* Test helper: (kf Cf, kr Cr) of every reaction [n][nR][2] at c = rho Y / W,
 * the gross forward and reverse rates that bound the rounding of the net ones. */
void orc_rate_parts(void* h, int nc, const double* rho, const double* y, double* out) {
    const mech_t* m = (const mech_t*)h;
    const int nS = m->nS, ne = nS + 2;
    double* c = (double*)malloc(sizeof(double) * (nS > 0 ? nS : 1));
    for (int j = 0; j < nc; ++j) {
        const double* yj = y + (size_t)j * ne;
        const double T = yj[nS];
        field_c(m, rho[j], yj, c);
        for (int r = 0; r < m->nR; ++r) {
            const rxn_t* R = &m->rx[r];
            const double clippedT = fmin(fmax(T, R->Tlow), R->Thigh);
            const double kf = rate_k(R, nS, clippedT, c);
            const double kr = R->irr ? 0.0 : kf / th_Kc(&R->th, clippedT);
            double Cf = 1.0, Cr = 1.0;
            for (int k = 0; k < R->nl; ++k) Cf *= specie_pow(c[R->lhs[k].index], &R->lhs[k]);
            for (int k = 0; k < R->nr; ++k) Cr *= specie_pow(c[R->rhs[k].index], &R->rhs[k]);
            out[((size_t)j * m->nR + r) * 2] = kf * Cf;
            out[((size_t)j * m->nR + r) * 2 + 1] = kr * Cr;
        }
    }
    free(c);
}

/* reactionRR(r) :188-229 (omega [n]) and specieReactionRR(r) :231-298 (RR [n][nS]) */
void orc_reaction_fields(void* h, int nc, int r, const double* rho, const double* y, double* omega, double* RR) {
    const mech_t* m = (const mech_t*)h;
    const int nS = m->nS, ne = nS + 2;
    const rxn_t* R = &m->rx[r];
    double* c = (double*)malloc(sizeof(double) * (nS > 0 ? nS : 1));
    for (int j = 0; j < nc; ++j) {
        const double* yj = y + (size_t)j * ne;
        field_c(m, rho[j], yj, c);
        const double om = rxn_omega(R, nS, yj[nS + 1], yj[nS], c);
        if (omega) omega[j] = om;
        if (RR) {
            double* o = RR + (size_t)j * nS;
            for (int i = 0; i < nS; ++i) o[i] = 0.0;
            for (int k = 0; k < R->nl; ++k) o[R->lhs[k].index] -= R->lhs[k].stoich * om;
            for (int k = 0; k < R->nr; ++k) o[R->rhs[k].index] += R->rhs[k].stoich * om;
            for (int i = 0; i < nS; ++i) o[i] = o[i] * m->th[i].W;
        }
    }
    free(c);
}

/* Qdot() :429-450: Qdot = 0 - sum_i hf_i RR_i in species order */
void orc_qdot(void* h, int nc, const double* RR, double* qdot) {
    const mech_t* m = (const mech_t*)h;
    for (int j = 0; j < nc; ++j) {
        double q = 0;
        for (int i = 0; i < m->nS; ++i) q -= th_Hf(&m->th[i]) * RR[(size_t)j * m->nS + i];
        qdot[j] = q;
    }
}

void orc_constants(double* out) {
    out[0] = ORC_RR;
    out[1] = ORC_PSTD;
    out[2] = ORC_TSTD;
    out[3] = 6.02214e+26;
    out[4] = 1.38065e-23;
    out[5] = ORC_VGREAT;
    out[6] = ORC_VSMALL;
    out[7] = ORC_SMALL;
    out[8] = ORC_GREAT;
}
