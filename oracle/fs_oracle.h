/* CPU oracle for the FARRSIGHT per-step hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * Plain C restatement of the reference (shujhan/multi_species) algorithm.  Each
 * function cites the reference file:line it follows.  Only tests/,
 * __graft_entry__.smoke() and the CPU-baseline leg of bench.py may load it; the
 * product library never links or calls it.
 *
 * Pinning: the field functions (fso_direct_sum, fso_treecode) are checked
 * against the reference's own src/FieldStructure.cpp compiled unmodified into
 * oracle/_ref/libfs_ref.so.  The mesh, remesh, RK4, step control, reduced
 * grid, adaptive refinement and initial conditions are checked bit for bit
 * against the reference's own AMRStructure / AMRSimulation sources compiled
 * into oracle/_ref/libamr_ref.so (with stand-ins for the Eigen and Boost calls
 * they make, oracle/refshim).  The 9x9 solve here and the Eigen stand-in use
 * the same partial-pivot LU; against Eigen itself the fits agree to rounding.
 */
#ifndef FS_ORACLE_H
#define FS_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------- field ---------------- */
/* E_MQ_DirectSum::operator() (src/FieldStructure.cpp:106-156). */
void fso_direct_sum(double L, double eps, double* es, const double* targets, int nt,
                    const double* sources, const double* q_ws, int ns);
/* E_MQ_Treecode::operator() (src/FieldStructure.cpp:230-503); targets ignored,
 * es[0..ns) written.  Returns the number of leaves (>0) or <0 on error. */
int fso_treecode(double L, double eps, double mac, int degree, int max_source,
                 double* es, const double* sources, const double* q_ws, int ns);

/* ---------------- mesh ---------------- */
/* Panel record exported as FSO_PANEL_INTS ints:
 * [0..8] point_inds, [9] level, [10] parent, [11] which_child, [12] child_start,
 * [13] left, [14] top, [15] right, [16] bottom,
 * [17] flags: 1 is_left_bdry, 2 is_right_bdry, 4 is_refined_xp, 8 is_refined_p */
#define FSO_PANEL_INTS 18
typedef struct fso_mesh fso_mesh;
/* create_prerefined_mesh (src/structure_files/AMRStructure_amr.cpp:127-230)
 * with refine_panels (:506-839) and refine_panels_refine_v (:233-504),
 * periodic boundary conditions, uniform refinement. */
fso_mesh* fso_mesh_build(int initial_height, int p_height, double xmin, double xmax,
                         double pmin, double pmax);
void fso_mesh_destroy(fso_mesh* m);
int fso_mesh_npoints(const fso_mesh* m);
int fso_mesh_npanels(const fso_mesh* m);
int fso_mesh_nleaves(const fso_mesh* m);
void fso_mesh_points(const fso_mesh* m, double* xs, double* ps);
void fso_mesh_panels(const fso_mesh* m, int* rec);
void fso_mesh_leaves(const fso_mesh* m, int* leaf_inds);
/* set_leaves_weights without the final *f (AMRStructure_amr.cpp:1084-1151):
 * w[i] = sum over leaves (DFS order) of q*dx*dp/{4,9} * stencil. quad 0 trap, 1 simpson */
void fso_mesh_base_weights(const fso_mesh* m, double q, int quad, double* w);

/* ---------------- initial conditions ---------------- */
/* src/structure_files/initial_distributions.cpp:16-140, ics_type 1,2,3,4,9,10 */
double fso_f0(int ics_type, double pth, double pstr, double k, double amp, double x, double p);

/* ---------------- remesh ---------------- */
/* interpolate_to_initial_xps (AMRStructure_interp.cpp:493-793) with shift_xs
 * (:429-491), the recursive first-point search (:232-426), the neighbour walk
 * (:12-230) and the per-panel 9x9 biquadratic fit (:795-975).
 * old_* are the deformed points of the previous mesh (same panel structure m);
 * new_fs receives f at the mesh lattice points (in mesh point order).
 * leaf_of_point / final_x (optional) receive the located leaf (0 = beyond the
 * p-boundary) and the periodically shifted x used for the fit.
 * Returns 0, or -1 when shift_xs needs more than 10 shifts (the reference throws). */
int fso_remesh_interp(const fso_mesh* m, const double* old_xs, const double* old_ps,
                      const double* old_fs, double f_beyond, double* new_fs,
                      int* leaf_of_point, double* final_x);
/* The same with the previous mesh's panels (old_m) distinct from the new base
 * mesh (new_m, uniform), as after an adaptive step: f at new_m's points. */
int fso_remesh_interp2(const fso_mesh* old_m, const fso_mesh* new_m, const double* old_xs, const double* old_ps,
                       const double* old_fs, double f_beyond, double* new_fs);
/* interpolate_from_mesh (AMRStructure_interp.cpp:1094-1143): f at one point from
 * the previous mesh -- shift_xs, the recursive search from the root, the leaf's
 * fit (f_beyond beyond the p-boundary).  *rc = -1 when shifting fails. */
double fso_interp_point(const fso_mesh* old_m, const double* old_xs, const double* old_ps, const double* old_fs,
                        double f_beyond, double x, double p, int* rc);

/* Adaptive refinement (generate_mesh, AMRStructure_amr.cpp:901-941; test_panel
 * :971-1081; refine_panels :506-839 on flagged panels).  f holds the values at
 * the mesh's current points; new points get theirs from eval(ctx, x, p, n, out).
 * Panels below max_height whose 9 values meet a criterion are split 2x2 until
 * none is flagged.  Returns the new f (realloc'ed, npoints entries). */
typedef void (*fso_eval_fn)(void* ctx, const double* x, const double* p, int n, double* out);
double* fso_mesh_adapt(fso_mesh* m, double* f, const double* amr_eps, int neps, int max_height, fso_eval_fn eval,
                       void* ctx);
/* One 9-point biquadratic fit evaluated at (dx, dp) offsets from point 4. */
void fso_panel_fit(const double* px, const double* py, const double* pf, int npts,
                   const double* x, const double* p, double* out);

/* ---------------- reduced grid ---------------- */
/* get_reduced_xs_ws (src/structure_files/AMRStructure.cpp:147-185): returns the
 * number of unique x; reduced_xs/ws sized n, inv sized n. */
int fso_reduce(const double* xs, const double* q_ws, int n, double* reduced_xs,
               double* reduced_ws, int* inv);

/* E_MQ_DirectSum_openbcs::operator() (src/FieldStructure.cpp:170-192):
 * open boundaries, es[i] = sum_j q_j 0.5 z / sqrt(z^2 + eps^2) - x_i. */
void fso_direct_sum_open(double eps, double* es, const double* targets, int nt, const double* sources,
                         const double* q_ws, int ns);

/* Drive fields (src/FieldStructure.cpp:15-96): amplitude at time t of
 * ExternalTanh (type 0, including its factor k), ExternalSine (1) and
 * ExternalLogistic (2); fso_external_field adds amp * sin(k x - omega t). */
double fso_external_amplitude(int type, double Am, double k, double t);
void fso_external_field(int type, double Am, double k, double omega, double* es, const double* x, int n,
                        double t);

/* ---------------- simulation ---------------- */
typedef struct {
    double q, m;
    int initial_height, p_height;
    double pmin, pmax;
    int ics_type;
    double pth, pstr, amp, normalized_wavenumber;
    /* adaptive refinement (AMRSimulation_load.cpp:246-258) */
    int do_adaptively_refine;
    int max_height;
    int n_amr_eps;              /* 0..5 */
    double amr_eps[5];
    /* "mu" of ics 6 and 7, "wave_beta" of ics 8 (AMRSimulation_load.cpp:169-207) */
    double mu, wave_beta;
} fso_species_params;

/* The distribution make_f0_return_ptr builds (AMRSimulation_load.cpp:139-225)
 * for every ics_type, with the Friedman-beam and travelling-wave tables.
 * fso_dist_create returns NULL and sets *rc when the parameters are invalid
 * (rc 1: argument; the reference throws or reads out of range there);
 * fso_dist_eval sets *rc = 1 where the reference would read past a table. */
typedef struct fso_dist fso_dist;
fso_dist* fso_dist_create(const fso_species_params* q, double xmin, double xmax, int* rc);
double fso_dist_eval(const fso_dist* d, double x, double p, int* rc);
void fso_dist_destroy(fso_dist* d);
/* Special functions of the relativistic initial conditions, restated from
 * their definitions: K_1 by the trapezoid rule on
 * int_0^inf exp(-x cosh t) cosh t dt, F and E by Carlson's symmetric
 * integrals R_F and R_D with the duplication theorem (B. C. Carlson, Numer.
 * Algorithms 10 (1995) 13-26) and F(k, phi + n pi) = F(k, phi) + 2 n K(k). */
double fso_bessel_k1(double x);
double fso_ellint_1(double k, double phi);
double fso_ellint_2(double k, double phi);

typedef struct {
    double xmin, xmax;
    int quadrature;      /* 0 trap, 1 simpson */
    double dt;
    int remesh_period;
    double greens_epsilon;
    int use_treecode;
    double mac;
    int degree;
    int max_source;
    int num_species;
    fso_species_params species[8];
    /* deck "external_field" (AMRSimulation_load.cpp:98-136) */
    int use_external_field;
    int external_type;   /* 0 tanh, 1 sine, 2 logistic */
    double ext_Am, ext_k, ext_omega;
    /* positions move with (p/m)/sqrt(1 + (p/m)^2) in every RK4 stage
     * (relativistic_momentum_push, AMRSimulation_step.cpp:101-111); 0 = the
     * reference's rk4_step, which moves them with p */
    int relativistic_push;
} fso_sim_params;

typedef struct fso_sim fso_sim;
/* AMRSimulation ctor (src/simulation_files/AMRSimulation.cpp:5-91): meshes,
 * f0, weights, initial reduced field. */
fso_sim* fso_sim_create(const fso_sim_params* prm);
void fso_sim_destroy(fso_sim* s);
/* AMRSimulation::step (src/simulation_files/AMRSimulation_step.cpp:5-99). */
int fso_sim_step(fso_sim* s);
int fso_sim_total_points(const fso_sim* s);
int fso_sim_species_points(const fso_sim* s, int sp);
int fso_sim_iter(const fso_sim* s);
/* Concatenated state (species in deck order). Any pointer may be NULL. */
void fso_sim_state(const fso_sim* s, double* xs, double* ps, double* fs, double* q_ws,
                   double* es);
/* Number of full (N x N) and reduced field evaluations done so far. */
void fso_sim_counters(const fso_sim* s, long long* full_evals, long long* reduced_evals);

#ifdef __cplusplus
}
#endif
#endif
