/*
 * libgrpp-compatible C API of the B200 GRPP integral engine.
 *
 * This header re-declares, in code written for this project, the public
 * interface of libgrpp that callers link against, so that this engine is a
 * drop-in replacement for it.  Struct layouts, names, argument order and
 * meaning are kept identical on purpose: a caller compiled against libgrpp's
 * own header must work unchanged against this library.
 *
 * Reference interface replaced (file:line within aoleynichenko/libgrpp):
 *   limits ................................ libgrpp/libgrpp.h:16-31
 *   init/finalize ......................... libgrpp/libgrpp.h:33-37, init_finalize.c:19-50
 *   libgrpp_potential_t + ctor/dtor ....... libgrpp/libgrpp.h:42-60, potential.c:22-115
 *   libgrpp_shell_t + ctor/dtor ........... libgrpp/libgrpp.h:66-88, shell.c:23-126
 *   libgrpp_grpp_t + builders ............. libgrpp/libgrpp.h:94-113, grpp.c:15-109
 *   integrators ........................... libgrpp/libgrpp.h:120-171
 *   gradients ............................. libgrpp/libgrpp.h:178-231
 *   overlap, kinetic, momentum ............ libgrpp/overlap.h, kinetic.h, momentum.h,
 *                                           overlap_gradient.h (libgrpp.h:237-241)
 *   nuclear attraction .................... libgrpp/libgrpp.h:243-310, nuclear_attraction.c:31-236
 *   nuclear charge models ................. libgrpp/nuclear_models.h:14-48
 *   parameters ............................ libgrpp/parameters.h:11-35
 *
 * All integrators return void, zero their outputs first, and write
 * cart_size(A) x cart_size(B) row-major blocks (matrix[i*size_B + j]).
 * Device faults and invalid input are reported through
 * libgrpp_b200_last_error() (declared in libgrpp_b200.h) instead of assert().
 */
#ifndef LIBGRPP_B200_LIBGRPP_H
#define LIBGRPP_B200_LIBGRPP_H

#ifdef __cplusplus
extern "C" {
#endif

/* maximum angular momentum of basis functions (libgrpp.h:16) */
#define LIBGRPP_MAX_BASIS_L 10
/* maximum angular momentum occurring in the RPP operator (libgrpp.h:21) */
#define LIBGRPP_MAX_RPP_L 10
/* threshold for zero (libgrpp.h:26) */
#define LIBGRPP_ZERO_THRESH 1e-14
/* tolerance of radial integrals evaluation (libgrpp.h:31) */
#define LIBGRPP_RADIAL_TOL 1e-14

/* ---- parameters (parameters.h:11-35) ---------------------------------- */
enum {
    LIBGRPP_CART_ORDER_DIRAC,
    LIBGRPP_CART_ORDER_TURBOMOLE
};

typedef struct {
    double radial_tolerance;
    double angular_screening_tolerance;
    double modified_bessel_tolerance;
    int (*cartesian_generator)(int L, int *cart_list);
} libgrpp_parameters_t;

extern libgrpp_parameters_t libgrpp_params;

void libgrpp_set_default_parameters(void);
void libgrpp_set_radial_tolerance(double tolerance);
void libgrpp_set_angular_screening_tolerance(double tolerance);
void libgrpp_set_modified_bessel_tolerance(double tolerance);
void libgrpp_set_cartesian_order(int order);
void libgrpp_set_cartesian_generator(int (*cartesian_generator)(int L, int *cart_list));

/* ---- init (libgrpp.h:33-37) ------------------------------------------- */
void libgrpp_init(void);
void libgrpp_finalize(void);
int libgrpp_is_initialized(void);

/* ---- potentials: sum_k c_k r^(n_k-2) exp(-alpha_k r^2) (libgrpp.h:42-60) */
typedef struct {
    int L;
    int J;
    int num_primitives;
    int *powers;
    double *coeffs;
    double *alpha;
} libgrpp_potential_t;

libgrpp_potential_t *libgrpp_new_potential(int L, int J, int num_primitives, int *powers,
                                           double *coeffs, double *alpha);
void libgrpp_delete_potential(libgrpp_potential_t *potential);
double libgrpp_potential_value(libgrpp_potential_t *potential, double r);
libgrpp_potential_t *libgrpp_shrink_potential(libgrpp_potential_t *src_potential);

/* ---- shells of contracted Cartesian Gaussians (libgrpp.h:66-88) -------- */
typedef struct {
    int L;
    int cart_size;
    int *cart_list;
    int num_primitives;
    double *coeffs;
    double *alpha;
    double origin[3];
} libgrpp_shell_t;

libgrpp_shell_t *libgrpp_new_shell(double *origin, int L, int num_primitives, double *coeffs,
                                   double *alpha);
int libgrpp_get_shell_size(libgrpp_shell_t *shell);
void libgrpp_delete_shell(libgrpp_shell_t *shell);
int *libgrpp_generate_shell_cartesians(int L);
libgrpp_shell_t *libgrpp_shell_deep_copy(libgrpp_shell_t *src_shell);
void libgrpp_shell_shrink(libgrpp_shell_t *shell);
void libgrpp_shell_mult_normcoef(libgrpp_shell_t *shell);

/* ---- the full GRPP operator of one element (libgrpp.h:94-113) ---------- */
typedef struct {
    int n_arep;
    int n_esop;
    int n_oc_shells;
    libgrpp_potential_t *U_L;
    libgrpp_potential_t **U_arep;
    libgrpp_potential_t **U_esop;
    libgrpp_potential_t **U_oc;
    libgrpp_shell_t **oc_shells;
} libgrpp_grpp_t;

libgrpp_grpp_t *libgrpp_new_grpp(void);
void libgrpp_grpp_set_local_potential(libgrpp_grpp_t *grpp, libgrpp_potential_t *pot);
void libgrpp_grpp_add_averaged_potential(libgrpp_grpp_t *grpp, libgrpp_potential_t *pot);
void libgrpp_grpp_add_spin_orbit_potential(libgrpp_grpp_t *grpp, libgrpp_potential_t *pot);
void libgrpp_grpp_add_outercore_potential(libgrpp_grpp_t *grpp, libgrpp_potential_t *pot,
                                          libgrpp_shell_t *oc_shell);
void libgrpp_delete_grpp(libgrpp_grpp_t *grpp);

/* ---- integrators (libgrpp.h:120-171) ----------------------------------- */
void libgrpp_type1_integrals(libgrpp_shell_t *shell_A, libgrpp_shell_t *shell_B,
                             double *rpp_origin, libgrpp_potential_t *potential, double *matrix);

void libgrpp_type2_integrals(libgrpp_shell_t *shell_A, libgrpp_shell_t *shell_B,
                             double *rpp_origin, libgrpp_potential_t *potential, double *matrix);

void libgrpp_spin_orbit_integrals(libgrpp_shell_t *shell_A, libgrpp_shell_t *shell_B,
                                  double *rpp_origin, libgrpp_potential_t *potential,
                                  double *so_x_matrix, double *so_y_matrix, double *so_z_matrix);

void libgrpp_outercore_potential_integrals(libgrpp_shell_t *shell_A, libgrpp_shell_t *shell_B,
                                           double *rpp_origin, int num_oc_shells,
                                           libgrpp_potential_t **oc_potentials,
                                           libgrpp_shell_t **oc_shells, double *arep,
                                           double *esop_x, double *esop_y, double *esop_z);

void libgrpp_full_grpp_integrals(libgrpp_shell_t *shell_A, libgrpp_shell_t *shell_B,
                                 libgrpp_grpp_t *grpp_operator, double *grpp_origin,
                                 double *arep_matrix, double *so_x_matrix, double *so_y_matrix,
                                 double *so_z_matrix);

/* ---- gradients w.r.t. the nuclear point point_3d (libgrpp.h:178-231) ---
 * grad_* are double*[3] (x, y, z), each cart_size(A) x cart_size(B). */
void libgrpp_type1_integrals_gradient(libgrpp_shell_t *shell_A, libgrpp_shell_t *shell_B,
                                      double *grpp_origin, libgrpp_potential_t *potential,
                                      double *point_3d, double **grad_arep);

void libgrpp_type2_integrals_gradient(libgrpp_shell_t *shell_A, libgrpp_shell_t *shell_B,
                                      double *grpp_origin, libgrpp_potential_t *potential,
                                      double *point_3d, double **grad_arep);

void libgrpp_spin_orbit_integrals_gradient(libgrpp_shell_t *shell_A, libgrpp_shell_t *shell_B,
                                           double *grpp_origin, libgrpp_potential_t *potential,
                                           double *point_3d, double **grad_so_x,
                                           double **grad_so_y, double **grad_so_z);

void libgrpp_outercore_potential_integrals_gradient(libgrpp_shell_t *shell_A,
                                                    libgrpp_shell_t *shell_B, double *rpp_origin,
                                                    int num_oc_shells,
                                                    libgrpp_potential_t **oc_potentials,
                                                    libgrpp_shell_t **oc_shells, double *point_3d,
                                                    double **grad_arep, double **grad_so_x,
                                                    double **grad_so_y, double **grad_so_z);

void libgrpp_full_grpp_integrals_gradient(libgrpp_shell_t *shell_A, libgrpp_shell_t *shell_B,
                                          libgrpp_grpp_t *grpp_operator, double *grpp_origin,
                                          double *point_3d, double **grad_arep,
                                          double **grad_so_x, double **grad_so_y,
                                          double **grad_so_z);

/* ---- other integrals (libgrpp.h:237-241) ------------------------------- */
/* <A|B> (overlap.h:13, overlap.c:39-62) */
void libgrpp_overlap_integrals(libgrpp_shell_t *shell_A, libgrpp_shell_t *shell_B, double *overlap_matrix);

/* d<A|B>/d point_3d, grad is double*[3] (overlap_gradient.h:13-18, overlap_gradient.c:27-82) */
void libgrpp_overlap_integrals_gradient(libgrpp_shell_t *shell_A, libgrpp_shell_t *shell_B, double *point_3d,
                                        double **grad);

/* <A| -1/2 nabla^2 |B> (kinetic.h:13, kinetic.c:34-57) */
void libgrpp_kinetic_energy_integrals(libgrpp_shell_t *shell_A, libgrpp_shell_t *shell_B, double *kinetic_matrix);

/* <A| d/dx |B>, <A| d/dy |B>, <A| d/dz |B> (momentum.h:13-19, momentum.c:34-68) */
void libgrpp_momentum_integrals(libgrpp_shell_t *shell_A, libgrpp_shell_t *shell_B, double *momentum_x_matrix,
                                double *momentum_y_matrix, double *momentum_z_matrix);

/* ---- nuclear attraction (libgrpp.h:243-310) ------------------------------ */
enum {
    LIBGRPP_NUCLEAR_MODEL_POINT_CHARGE = 0,
    LIBGRPP_NUCLEAR_MODEL_CHARGED_BALL,
    LIBGRPP_NUCLEAR_MODEL_GAUSSIAN,
    LIBGRPP_NUCLEAR_MODEL_FERMI,
    LIBGRPP_NUCLEAR_MODEL_FERMI_BUBBLE,
    LIBGRPP_NUCLEAR_MODEL_POINT_CHARGE_NUMERICAL
};

/* <A| V_nuc(|r - C|) |B> of a nucleus of charge Z at charge_origin; model_params: ball and
 * Gaussian {R_rms}, Fermi {c, a}, Fermi bubble {c, a, k}, NULL for point charges
 * (nuclear_attraction.c:31-119) */
void libgrpp_nuclear_attraction_integrals(libgrpp_shell_t *shell_A, libgrpp_shell_t *shell_B, double *charge_origin,
                                          int charge, int nuclear_model, double *model_params, double *coulomb_matrix);

/* The model-specific forms below pass libgrpp_nuclear_attraction_integrals the array
 * {charge, parameters...}, as libgrpp's do (nuclear_attraction.c:177-236); the generic function
 * reads the model's parameters from the first element, so these forms use the charge as the
 * first model parameter, exactly as in libgrpp. */
void libgrpp_nuclear_attraction_integrals_point_charge(libgrpp_shell_t *shell_A, libgrpp_shell_t *shell_B,
                                                       double *charge_origin, int charge, double *coulomb_matrix);

void libgrpp_nuclear_attraction_integrals_charged_ball(libgrpp_shell_t *shell_A, libgrpp_shell_t *shell_B,
                                                       double *charge_origin, int charge, double r_rms,
                                                       double *coulomb_matrix);

void libgrpp_nuclear_attraction_integrals_gaussian_model(libgrpp_shell_t *shell_A, libgrpp_shell_t *shell_B,
                                                         double *charge_origin, int charge, double r_rms,
                                                         double *coulomb_matrix);

void libgrpp_nuclear_attraction_integrals_fermi_model(libgrpp_shell_t *shell_A, libgrpp_shell_t *shell_B,
                                                      double *charge_origin, int charge, double fermi_param_c,
                                                      double fermi_param_a, double *coulomb_matrix);

void libgrpp_nuclear_attraction_integrals_fermi_bubble_model(libgrpp_shell_t *shell_A, libgrpp_shell_t *shell_B,
                                                             double *charge_origin, int charge, double param_c,
                                                             double param_a, double param_k, double *coulomb_matrix);

/* ---- nuclear charge models (nuclear_models.h:14-48) ------------------------ */
#define FERMI_UNITS_TO_ATOMIC (1.0 / 52917.7210903)

double libgrpp_estimate_nuclear_rms_radius_johnson_1985(int A);
double libgrpp_estimate_nuclear_rms_radius_golovko_2008(int A);
int libgrpp_estimate_fermi_model_parameters(double R_rms, double *c, double *a);
double libgrpp_charge_density_ball(double r, double Z, double R_rms);
double libgrpp_charge_density_gaussian(double r, double Z, double R_rms);
double libgrpp_charge_density_fermi(double r, double Z, double c, double a);
double libgrpp_charge_density_fermi_bubble(double r, double Z, double c, double a, double k);
double libgrpp_rms_radius_fermi(int Z, double c, double a);
double libgrpp_rms_radius_fermi_bubble(int Z, double c, double a, double k);
double libgrpp_coulomb_potential_point(double r, double Z);
double libgrpp_coulomb_potential_ball(double r, double Z, double R_rms);
double libgrpp_coulomb_potential_gaussian(double r, double Z, double R_rms);
double libgrpp_coulomb_potential_fermi(double r, double Z, double c, double a);
double libgrpp_coulomb_potential_fermi_bubble(double r, double Z, double c, double a, double k);

#ifdef __cplusplus
}
#endif

#endif /* LIBGRPP_B200_LIBGRPP_H */
