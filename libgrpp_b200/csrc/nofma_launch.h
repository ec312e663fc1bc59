// Launches of the kernels that must round as libgrpp does: the angular tensors (atab_kernel),
// the outercore spherical projections (oc_proj_kernel), the omega tables (omega_tab_kernel),
// the per-task assembly (final_kernel) and the radial integrand tables, F_l(r) per (shell,
// centre) pair (ftab_kernel) and w U_p(r) per GRPP (wu_table_kernel).
//
// These kernels live in their own translation unit, nofma.cu, compiled without
// floating-point contraction (nvcc -fmad=false). libgrpp is plain C built without FMA
// contraction, so every a*b + c in its angular sums, binomial re-centring, outercore products,
// Bessel Taylor series and contracted integrands is a rounded multiply followed by a rounded
// add (type2_integrals.c:129-205, spin_orbit_integrals.c:150-243, angular_integrals.c:63-108,
// outercore_integrals.c:147-390, specfunc_scaled_mod_sph_bessel.c:94-118,
// radial_type2_integral.c:465-481). On elements where the re-centring sum cancels by many
// orders of magnitude (high-l shells a few bohr from the potential centre) a fused
// multiply-add anywhere on that path changes the result far above libgrpp's 1e-10
// comparator, so these values are evaluated with libgrpp's rounding.
//
// The argument structs (FinalArgs, FinalSmem, OcProjArgs, DeviceTables) are those of
// angular.cuh, radial.cuh and grpp_common.cuh; they are passed by address with their size, which the
// launch functions check against their own definition of the same structs.
#pragma once

#include <cstddef>
#include <cuda_runtime.h>

namespace grpp {

// copies the device table descriptor (DeviceTables) into this unit's constant memory
cudaError_t ang_upload_tables(const void *tables, size_t size);
// maximum dynamic shared memory of the assembly kernel at every block size
cudaError_t ang_set_final_max_smem(int bytes);
cudaError_t ang_final_occupancy(int nt, size_t smem, int *blocks_per_sm);
cudaError_t ang_launch_atab(int blocks, int threads, cudaStream_t s, int L, int l, double *out);
cudaError_t ang_launch_oc_proj(int blocks, int threads, cudaStream_t s, const void *args, size_t size);
cudaError_t ang_launch_omega_tab(int blocks, int threads, size_t smem, cudaStream_t s, const void *fin, size_t fin_size,
                                 const void *layout, size_t layout_size, const int *op_shell, const int *op_centre,
                                 int n_pairs, double *omtab);
// RadialArgs (radial.cuh) by address and size
cudaError_t nofma_launch_ftab(int blocks, int threads, size_t smem, cudaStream_t s, const void *rad, size_t rad_size,
                              double *ftab);
cudaError_t nofma_launch_wu_table(int blocks, int threads, cudaStream_t s, const void *rad, size_t rad_size, int n_grpps,
                                  double *wu);
// nt = 128, 256 or 512 threads per block
cudaError_t ang_launch_final(int nt, int blocks, size_t smem, cudaStream_t s, const void *fin, size_t fin_size,
                             const void *layout, size_t layout_size);

}  // namespace grpp
