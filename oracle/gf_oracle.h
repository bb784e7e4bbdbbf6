/*
 * TEST INFRASTRUCTURE ONLY — the CPU oracle of this project.
 *
 * A plain-C restatement of gpuFoam's per-cell chemistry path (reaction rates,
 * analytic Jacobian, Crout LU, Rosenbrock12/23/34 with adaptive step control,
 * the single-cell driver and the host computeRR arithmetic). It exists to check
 * the CUDA kernels; nothing in the product links or calls it.
 *
 * Parity pin: every function here is checked bit for bit against the
 * reference's own code compiled on the CPU (oracle/ref_driver.cpp, built by
 * oracle/Makefile into oracle/_ref/) and against the golden fixtures in
 * tests/golden/ that were generated from it.
 *
 * Flat raw mechanism format (shared with ref_driver.cpp):
 *   species: W, Tlow, Thigh, Tcommon [nS]; high_raw, low_raw [nS][7] (NASA-7
 *            coefficients before the x R scaling)
 *   reactions: rint [nR][24] = rate_type, irreversible, n_lhs, n_rhs,
 *              lhs index[10], rhs index[10];
 *              rdbl [nR][50] = lhs stoich[10], lhs exponent[10], rhs stoich[10],
 *              rhs exponent[10], A, beta, Ta, Ainf, betainf, Tainf,
 *              alpha, Tsss, Ts, Tss;
 *              eff [nR][nS] third-body efficiencies (read for rate types 1-3)
 */
#ifndef GF_ORACLE_H
#define GF_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_ode_inputs {  /* same layout as gf_ode_inputs */
    int solver;
    double absTol, relTol;
    int maxSteps;
    double safeScale, alphaInc, alphaDec, minScale, maxScale;
} orc_ode_inputs;

void* orc_mech_create(int nS, const double* W, const double* Tlow, const double* Thigh,
                      const double* Tcommon, const double* high_raw, const double* low_raw,
                      int nR, const int* rint, const double* rdbl, const double* eff,
                      double rxnTlow, double rxnThigh);
void orc_mech_destroy(void* h);
void orc_mech_tables(void* h, double* species_out, double* reaction_out, int* int_exp_out);
void orc_thermo_eval(void* h, double p, double T, double* out);
void orc_reaction_eval(void* h, const double* y, double* out);
void orc_derivatives(void* h, int n, const double* y, double* dydx);
void orc_jacobian(void* h, int n, const double* y, double* dfdx, double* J);
void orc_lu(int m, int n_mats, double* A, int* piv, double* b);
void orc_attempt(void* h, const orc_ode_inputs* o, int n, const double* y0, const double* dydx0,
                 const double* dx, double* y, double* err);
void orc_replay(void* h, const orc_ode_inputs* o, int n_steps, const double* steps, double* y);
void orc_cells(void* h, const orc_ode_inputs* o, double Treact, int n, double deltaT,
               const double* deltaT_cell, double* Y, double* deltaTChem, int* counts,
               int* status, int nthreads);
double orc_compute_rr_host(int n, int nS, double deltaT, double deltaTChemMax, const double* rho,
                           const double* Y0, const double* Ynew, double* deltaTChemNew, double* RR);
void orc_constants(double* out);
void orc_cell_fields(void* h, int n, const double* rho, const double* y, double* RR, double* tc);
void orc_reaction_fields(void* h, int n, int reaction, const double* rho, const double* y, double* omega,
                         double* RR);
void orc_qdot(void* h, int n, const double* RR, double* qdot);
void orc_rate_parts(void* h, int n, const double* rho, const double* y, double* out);

#ifdef __cplusplus
}
#endif
#endif
