// Krylov solve, excitation and far field on the device.
#pragma once
#include <vector>

#include "plan.hpp"

namespace mlfma {

struct SolveStats {
  int iterations = 0;
  int restarts = 0;
  int matvecs = 0;
  int near_products = 0;
  double rel_residual = 0.0;
  double seconds = 0.0;
};

// Restarted GMRES(mr) of Code/GMRES.h:65-217 on the device operator; x, rhs
// host complex128 [2N]. Returns true when converged.
bool gmres_solve(Plan& P, double* x, const double* rhs, int itr_max, int mr, double tol_abs, double tol_rel,
                 SolveStats& st, std::vector<double>& history);

// Flexible GMRES(mr) whose right preconditioner is inner_its GMRES steps on
// the near-field matrix alone (fgmres.cu); inner_its = 0 gives plain GMRES.
// prec 1: the operator and near field are the plan's complex64 copies (the
// Krylov vectors and Gram-Schmidt stay complex128).
bool fgmres_solve(Plan& P, double* x, const double* rhs, int itr_max, int mr, double tol_abs, double tol_rel,
                  int inner_its, SolveStats& st, std::vector<double>& history, int prec = 0);

// Mixed precision: FP64 iterative refinement (mixed.cu). Each step solves the
// correction equation A d = r with the complex64 operator (fgmres_solve,
// prec 1) to a relative tolerance that aims at tol_rel, then recomputes the
// residual r = b - A x with the FP64 operator. history: the FP64 relative
// residual after each refinement step.
bool mixed_solve(Plan& P, double* x, const double* rhs, int itr_max, int mr, double tol_abs, double tol_rel,
                 int inner_its, int refine_max, SolveStats& st, std::vector<double>& history);

// Lockstep FGMRES of R systems (fgmres_batch.cu): x, rhs host complex128
// [R][2N]; per system the iteration of fgmres_solve, with every operator
// apply and near-field product batched over the systems still iterating.
// Returns the converged flag of each system.
std::vector<char> fgmres_batch_solve(Plan& P, int R, double* x, const double* rhs, int itr_max, int mr,
                                     double tol_abs, double tol_rel, int inner_its, std::vector<SolveStats>& st,
                                     std::vector<std::vector<double>>& hist, double& seconds, int prec = 0);

// mixed_solve for R systems: FP64 residuals by batched applies, corrections
// by fgmres_batch_solve with the complex64 operator.
std::vector<char> mixed_batch_solve(Plan& P, int R, double* x, const double* rhs, int itr_max, int mr,
                                    double tol_abs, double tol_rel, int inner_its, int refine_max,
                                    std::vector<SolveStats>& st, double& seconds);

// w = Z_near x on device vectors (complex128 [2N]).
void near_apply(Plan& P, const double2* x, double2* w, cudaStream_t s, int prec = 0);

// z = the near-field preconditioner applied to v (inner_its GMRES steps from
// zero on the complex64 Z_near, as inside fgmres_solve); device vectors,
// synchronous.
void near_precondition(Plan& P, int inner_its, const double2* v, double2* z, cudaStream_t s);

void rhs_pmchwt(Plan& P, const double kinc[3], const double einc[3], const double hinc[3], double* V);

void rcs_pmchwt(Plan& P, const double* I, int n_angles, const double* theta_deg, const double* phi_deg,
                double* field, double* rcs_db);

// Far field on device-resident currents and output without any device
// allocation: the angle table lives in a fixed file-scope device array of
// rcs_noalloc_max_angles() entries (see solver.cu).
void rcs_pmchwt_noalloc(Plan& P, const double2* I_dev, int n_angles, const double* theta_deg,
                        const double* phi_deg, double2* field_dev, cudaStream_t s);
int rcs_noalloc_max_angles();

// Many incidences at once (excitation.cu): the excitation vectors of R plane
// waves (host tables [R][3]) into V_dev [R][2N]; the far field of R current
// vectors I_dev [R][2N] at n_angles directions into field_dev
// [R][n_angles][3] (bistatic) or each at its own direction into [R][3]
// (monostatic). Asynchronous on s; the host tables are read at launch.
void rhs_pmchwt_batch(Plan& P, int R, const double* kinc, const double* einc, const double* hinc, double2* V_dev,
                      cudaStream_t s);
void rcs_pmchwt_batch(Plan& P, int R, const double2* I_dev, int n_angles, const double* theta_deg,
                      const double* phi_deg, double2* field_dev, cudaStream_t s);
void rcs_pmchwt_mono(Plan& P, int R, const double2* I_dev, const double* theta_deg, const double* phi_deg,
                     double2* field_dev, cudaStream_t s);
// dB of far fields (6 doubles per angle) as the reference forms them:
// total, theta-pol, phi-pol per angle.
void rcs_db(int n_angles, const double* theta_deg, const double* phi_deg, const double* field, double* out);

}  // namespace mlfma
