/*
 * Fortran ABI of the B200 GRPP integral engine.
 *
 * The symbols libgrpp's Fortran interface binds (libgrpp/fortran.c:29-1083): the
 * lower-case names with a trailing underscore that gfortran and ifort generate for
 * external procedures, every argument passed by address, integers as 32-bit. A Fortran
 * program linked against libgrpp's Fortran wrappers links against this library
 * unchanged (see test_libgrpp_f90/ for the caller's side). Each call builds libgrpp
 * objects from its arguments and evaluates the integrals on the GPU through the C API
 * of libgrpp.h; outputs are column-major from Fortran's point of view exactly as in
 * libgrpp (row-major cart(A) x cart(B) blocks in C terms).
 */
#ifndef LIBGRPP_B200_F90_H
#define LIBGRPP_B200_F90_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* parameters, initialisation (fortran.c:29-71) */
void libgrpp_set_default_parameters_(void);
void libgrpp_set_radial_tolerance_(const double *tolerance);
void libgrpp_set_angular_screening_tolerance_(const double *tolerance);
void libgrpp_set_modified_bessel_tolerance_(const double *tolerance);
void libgrpp_set_cartesian_order_(const int32_t *order);
void libgrpp_init_(void);
void libgrpp_finalize_(void);

/* type 1 (fortran.c:78-119): shells A, B by (origin, L, n, coeffs, alpha); potential (origin, n, powers, coeffs, alpha) */
void libgrpp_type1_integrals_(double *origin_A, int32_t *L_A, int32_t *num_primitives_A, double *coeffs_A, double *alpha_A,
                              double *origin_B, int32_t *L_B, int32_t *num_primitives_B, double *coeffs_B, double *alpha_B,
                              double *rpp_origin, int32_t *rpp_num_primitives, int32_t *rpp_powers, double *rpp_coeffs,
                              double *rpp_alpha, double *matrix);

/* type 2 (fortran.c:124-167) */
void libgrpp_type2_integrals_(double *origin_A, int32_t *L_A, int32_t *num_primitives_A, double *coeffs_A, double *alpha_A,
                              double *origin_B, int32_t *L_B, int32_t *num_primitives_B, double *coeffs_B, double *alpha_B,
                              double *pot_origin, int32_t *pot_L, int32_t *pot_num_primitives, int32_t *pot_powers,
                              double *pot_coeffs, double *pot_alpha, double *matrix);

/* spin-orbit (fortran.c:172-224) */
void libgrpp_spin_orbit_integrals_(double *origin_A, int32_t *L_A, int32_t *num_primitives_A, double *coeffs_A,
                                   double *alpha_A, double *origin_B, int32_t *L_B, int32_t *num_primitives_B,
                                   double *coeffs_B, double *alpha_B, double *pot_origin, int32_t *pot_L,
                                   int32_t *pot_num_primitives, int32_t *pot_powers, double *pot_coeffs, double *pot_alpha,
                                   double *so_x_matrix, double *so_y_matrix, double *so_z_matrix);

/* outercore part 1, U|nlj><nlj| + |nlj><nlj|U of one outercore shell (fortran.c:231-318) */
void libgrpp_outercore_potential_integrals_part_1_(double *origin_A, int32_t *L_A, int32_t *num_primitives_A,
                                                   double *coeffs_A, double *alpha_A, double *origin_B, int32_t *L_B,
                                                   int32_t *num_primitives_B, double *coeffs_B, double *alpha_B,
                                                   double *pot_origin, int32_t *pot_L, int32_t *pot_J,
                                                   int32_t *pot_num_primitives, int32_t *pot_powers, double *pot_coeffs,
                                                   double *pot_alpha, int32_t *oc_shell_num_primitives,
                                                   double *oc_shell_coeffs, double *oc_shell_alpha, double *arep_matrix,
                                                   double *so_x_matrix, double *so_y_matrix, double *so_z_matrix);

/* outercore part 2, |nlj><nlj| U |n'lj><n'lj| of a pair of outercore shells (fortran.c:325-436) */
void libgrpp_outercore_potential_integrals_part_2_(
    double *origin_A, int32_t *L_A, int32_t *num_primitives_A, double *coeffs_A, double *alpha_A, double *origin_B,
    int32_t *L_B, int32_t *num_primitives_B, double *coeffs_B, double *alpha_B, double *pot_origin, int32_t *oc_shell_1_L,
    int32_t *oc_shell_1_J, int32_t *pot1_num_primitives, int32_t *pot1_powers, double *pot1_coeffs, double *pot1_alpha,
    int32_t *oc_shell_1_num_primitives, double *oc_shell_1_coeffs, double *oc_shell_1_alpha, int32_t *oc_shell_2_L,
    int32_t *oc_shell_2_J, int32_t *pot2_num_primitives, int32_t *pot2_powers, double *pot2_coeffs, double *pot2_alpha,
    int32_t *oc_shell_2_num_primitives, double *oc_shell_2_coeffs, double *oc_shell_2_alpha, double *arep_matrix,
    double *so_x_matrix, double *so_y_matrix, double *so_z_matrix);

/* gradients w.r.t. point_3d (fortran.c:443-634) */
void libgrpp_type1_integrals_gradient_(double *origin_A, int32_t *L_A, int32_t *num_primitives_A, double *coeffs_A,
                                       double *alpha_A, double *origin_B, int32_t *L_B, int32_t *num_primitives_B,
                                       double *coeffs_B, double *alpha_B, double *rpp_origin, int32_t *rpp_num_primitives,
                                       int32_t *rpp_powers, double *rpp_coeffs, double *rpp_alpha, double *point_3d,
                                       double *grad_arep_x, double *grad_arep_y, double *grad_arep_z);

void libgrpp_type2_integrals_gradient_(double *origin_A, int32_t *L_A, int32_t *num_primitives_A, double *coeffs_A,
                                       double *alpha_A, double *origin_B, int32_t *L_B, int32_t *num_primitives_B,
                                       double *coeffs_B, double *alpha_B, double *pot_origin, int32_t *pot_L,
                                       int32_t *pot_num_primitives, int32_t *pot_powers, double *pot_coeffs,
                                       double *pot_alpha, double *point_3d, double *grad_arep_x, double *grad_arep_y,
                                       double *grad_arep_z);

void libgrpp_spin_orbit_integrals_gradient_(double *origin_A, int32_t *L_A, int32_t *num_primitives_A, double *coeffs_A,
                                            double *alpha_A, double *origin_B, int32_t *L_B, int32_t *num_primitives_B,
                                            double *coeffs_B, double *alpha_B, double *pot_origin, int32_t *pot_L,
                                            int32_t *pot_num_primitives, int32_t *pot_powers, double *pot_coeffs,
                                            double *pot_alpha, double *point_3d, double *grad_sox_x, double *grad_sox_y,
                                            double *grad_sox_z, double *grad_soy_x, double *grad_soy_y, double *grad_soy_z,
                                            double *grad_soz_x, double *grad_soz_y, double *grad_soz_z);

/* auxiliary overlap of single Cartesian components and radial norm (fortran.c:641-703) */
void evaluate_overlap_integral_contracted_(double *origin_A, int32_t *n_A, int32_t *l_A, int32_t *m_A,
                                           int32_t *num_primitives_A, double *coeffs_A, double *alpha_A, double *origin_B,
                                           int32_t *n_B, int32_t *l_B, int32_t *m_B, int32_t *num_primitives_B,
                                           double *coeffs_B, double *alpha_B, double *overlap_integral);
void radial_gto_norm_factor_(int32_t *L, int32_t *num_primitives, double *coeffs, double *alpha, double *norm);

/* overlap, kinetic energy, momentum (fortran.c:709-797) */
void libgrpp_overlap_integrals_(double *origin_A, int32_t *L_A, int32_t *num_primitives_A, double *coeffs_A,
                                double *alpha_A, double *origin_B, int32_t *L_B, int32_t *num_primitives_B,
                                double *coeffs_B, double *alpha_B, double *matrix);
void libgrpp_kinetic_energy_integrals_(double *origin_A, int32_t *L_A, int32_t *num_primitives_A, double *coeffs_A,
                                       double *alpha_A, double *origin_B, int32_t *L_B, int32_t *num_primitives_B,
                                       double *coeffs_B, double *alpha_B, double *matrix);
void libgrpp_momentum_integrals_(double *origin_A, int32_t *L_A, int32_t *num_primitives_A, double *coeffs_A,
                                 double *alpha_A, double *origin_B, int32_t *L_B, int32_t *num_primitives_B,
                                 double *coeffs_B, double *alpha_B, double *matrix_x, double *matrix_y, double *matrix_z);

/* nuclear attraction (fortran.c:804-993) */
void libgrpp_nuclear_attraction_integrals_(double *origin_A, int32_t *L_A, int32_t *num_primitives_A, double *coeffs_A,
                                           double *alpha_A, double *origin_B, int32_t *L_B, int32_t *num_primitives_B,
                                           double *coeffs_B, double *alpha_B, double *charge_origin, int32_t *charge,
                                           int32_t *nuclear_model, double *model_params, double *matrix);
void libgrpp_nuclear_attraction_integrals_point_charge_(double *origin_A, int32_t *L_A, int32_t *num_primitives_A,
                                                        double *coeffs_A, double *alpha_A, double *origin_B,
                                                        int32_t *L_B, int32_t *num_primitives_B, double *coeffs_B,
                                                        double *alpha_B, double *charge_origin, int32_t *charge,
                                                        double *matrix);
void libgrpp_nuclear_attraction_integrals_charged_ball_(double *origin_A, int32_t *L_A, int32_t *num_primitives_A,
                                                        double *coeffs_A, double *alpha_A, double *origin_B,
                                                        int32_t *L_B, int32_t *num_primitives_B, double *coeffs_B,
                                                        double *alpha_B, double *charge_origin, int32_t *charge,
                                                        double *r_rms, double *matrix);
void libgrpp_nuclear_attraction_integrals_gaussian_model_(double *origin_A, int32_t *L_A, int32_t *num_primitives_A,
                                                          double *coeffs_A, double *alpha_A, double *origin_B,
                                                          int32_t *L_B, int32_t *num_primitives_B, double *coeffs_B,
                                                          double *alpha_B, double *charge_origin, int32_t *charge,
                                                          double *r_rms, double *matrix);
void libgrpp_nuclear_attraction_integrals_fermi_model_(double *origin_A, int32_t *L_A, int32_t *num_primitives_A,
                                                       double *coeffs_A, double *alpha_A, double *origin_B, int32_t *L_B,
                                                       int32_t *num_primitives_B, double *coeffs_B, double *alpha_B,
                                                       double *charge_origin, int32_t *charge, double *fermi_param_c,
                                                       double *fermi_param_a, double *matrix);
void libgrpp_nuclear_attraction_integrals_fermi_bubble_model_(double *origin_A, int32_t *L_A, int32_t *num_primitives_A,
                                                              double *coeffs_A, double *alpha_A, double *origin_B,
                                                              int32_t *L_B, int32_t *num_primitives_B, double *coeffs_B,
                                                              double *alpha_B, double *charge_origin, int32_t *charge,
                                                              double *fermi_param_c, double *fermi_param_a,
                                                              double *param_k, double *matrix);

/* nuclear charge models (fortran.c:1000-1083) */
void libgrpp_estimate_nuclear_rms_radius_johnson_1985_(int32_t *A, double *R_rms);
void libgrpp_estimate_nuclear_rms_radius_golovko_2008_(int32_t *A, double *R_rms);
void libgrpp_estimate_fermi_model_parameters_(double *R_rms, double *c, double *a, int32_t *err_code);
void libgrpp_charge_density_ball_(double *r, double *Z, double *R_rms, double *rho);
void libgrpp_charge_density_gaussian_(double *r, double *Z, double *R_rms, double *rho);
void libgrpp_charge_density_fermi_(double *r, double *Z, double *c, double *a, double *rho);
void libgrpp_charge_density_fermi_bubble_(double *r, double *Z, double *c, double *a, double *k, double *rho);
void libgrpp_coulomb_potential_point_(double *r, double *Z, double *potential);
void libgrpp_coulomb_potential_ball_(double *r, double *Z, double *R_rms, double *potential);
void libgrpp_coulomb_potential_gaussian_(double *r, double *Z, double *R_rms, double *potential);
void libgrpp_coulomb_potential_fermi_(double *r, double *Z, double *c, double *a, double *potential);
void libgrpp_coulomb_potential_fermi_bubble_(double *r, double *Z, double *c, double *a, double *k, double *potential);
void libgrpp_rms_radius_fermi_(int32_t *Z, double *c, double *a, double *r_rms);
void libgrpp_rms_radius_fermi_bubble_(int32_t *Z, double *c, double *a, double *k, double *r_rms);

#ifdef __cplusplus
}
#endif

#endif /* LIBGRPP_B200_F90_H */
