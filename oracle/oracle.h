/* Test infrastructure only: the C interface of the CPU oracle (a restatement of the reference's
 * CPU solvers; see flexure.cpp, diffusion.cpp and cube.cpp for the file:line each function follows). Only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load liboracle.so. */
#ifndef DEEPTIME_ORACLE_H
#define DEEPTIME_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

enum { DTO_PRECOND_REFERENCE = 0, DTO_PRECOND_MEAN_D = 1 };
enum { DTO_STOP_MAX_Z = 0, DTO_STOP_REL_RESIDUAL = 1, DTO_STOP_RMS_RESIDUAL = 2 };
enum { DTO_CYCLE_JACOBI = 0, DTO_CYCLE_RBGS = 1 };

typedef struct {
  int iterations;
  int converged;
  double error_m;      /* the reference's estimate: max |z| of the last preconditioned residual */
  double rel_residual; /* ||r||_2 / ||b||_2 of the recurrence residual at exit */
} dto_report;

void dto_set_threads(int n);
int dto_threads(void);
double dto_rigidity_per_g(double te_km, double g);
double dto_flexural_parameter_m(double d_per_g);
int dto_flex_spectral_roundtrip(int w, int h, double dx, const double* v, double* out);
int dto_flex_operator(int w, int h, double dx, const double* ma, const double* mb, const double* d, const double* c,
                      const double* v, double* y);
int dto_flex_bend(int w, int h, double dx, const double* d, const double* v, double* y);
int dto_flex_precondition(int w, int h, double dx, const double* ma, const double* mb, const double* d, const double* c,
                          const double* r, double* z, int precond);
int dto_flex_bank(int w, int h, double dx, const double* d, const double* c, double* node_d, double* c_ref, double* weights);
int dto_flex_solve(int w, int h, double dx, const double* ma, const double* mb, const double* d, const double* c, const double* b,
                   double* x, double tol, int max_it, int precond, int stop, dto_report* rep);
void dto_row_metric_from_sin_faces(const double* sin_faces, int nfaces, int f, double* a, double* b);
void dto_box_blur(int w, int h, int wrap, double* v, int r, int passes);
void dto_restrict_by(int w, int h, int f, const double* v, double* out);
void dto_prolong_const(int ws, int hs, int f, const double* v, double* out);
void dto_prolong_linear(int ws, int hs, int f, const double* v, double* out);
void dto_binomial(int w, int h, int passes, double* v);

/* The cube grid's diffusion (surface/cube/diffusion.rs, surface/cube/multigrid.rs): slots are
 * 6 n^2 x 8 neighbour indices (0xFFFFFFFF: none), lap 6 n^2 x 8 coupling weights, areas 6 n^2. */
void dto_cube_topology(int n, uint32_t* slots);
void dto_cube_operator(int n, const uint32_t* slots, const double* lap, const double* areas, const double* kd, double dt,
                       const double* x, double* y);
void dto_cube_vcycle(int n, const uint32_t* slots, const double* lap, const double* areas, const double* kd, double dt,
                     const double* r, double* z);
void dto_cube_lod(int n, const uint32_t* slots, const double* lap, const double* areas, const double* kd, double dt,
                  const double* h, double* x);
int dto_cube_diff_solve(int n, const uint32_t* slots, const double* lap, const double* areas, const double* kd, double dt,
                        double tol_m, double* h);

int dto_diff_operator(int w, int h, double dx, int wrap, const double* kd, double dt, const double* x, double* y);
int dto_diff_operator_coeffs(int w, int h, double dx, int wrap, const double* kd, double dt, double* east, double* south,
                             double* diag);
int dto_diff_apply_reference(int w, int h, double dx, int wrap, const double* kd, double dt, const double* x, double* y);
int dto_diff_lod(int w, int h, double dx, int wrap, double* hfield, const double* kd, double dt);
void dto_thomas(const double* lo, const double* di, const double* up, double* b, int n);
void dto_cyclic(const double* lo, const double* di, const double* up, double alpha, double beta, double* b, int n);
int dto_diff_solve_jacobi(int w, int h, double dx, int wrap, double* hfield, const double* kd, double dt, int use_lod);
int dto_diff_solve_mg(int w, int h, double dx, int wrap, double* hfield, const double* kd, double dt, double tol, int stop,
                      int cycle, int precision, int use_lod, int max_it, double* rel_res);
double dto_diff_vcycle(int w, int h, double dx, int wrap, const double* kd, double dt, int cycle, const double* r, float* z,
                       int* levels_out);
int dto_diff_reference_cg(int w, int h, double dx, int wrap, const double* b, const double* kd, double dt, double rel,
                          double* x);
double dto_submarine_kd(double z, double d0, double wave_base, double tidal_range, double land);

#ifdef __cplusplus
}
#endif
#endif
