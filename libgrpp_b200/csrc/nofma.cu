// Translation unit of the kernels that round as libgrpp does (nofma_launch.h): the angular-part
// kernels of angular.cuh and the radial integrand tables of radial.cuh, compiled with
// -fmad=false. The kernel headers are included
// in a namespace of their own, as in noalloc.cu, so this unit's constant table descriptor
// and kernels do not clash with engine.cu's; engine.cu reaches them through the launch
// functions below.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>

#include "nofma_launch.h"

#define GRPP_RADIAL_TABLES_ONLY  // of radial.cuh only the integrand-table kernels
namespace grpp_ang {
#include "grpp_common.cuh"
#include "specfunc.cuh"
#include "radial.cuh"
#include "angular.cuh"
}  // namespace grpp_ang

namespace grpp {

namespace {
using AFin = grpp_ang::grpp::FinalArgs;
using ASmem = grpp_ang::grpp::FinalSmem;
using AOcp = grpp_ang::grpp::OcProjArgs;
using ATab = grpp_ang::grpp::DeviceTables;
using ARad = grpp_ang::grpp::RadialArgs;

template <class T>
bool unpack(T &dst, const void *src, size_t size)
{
    if (size != sizeof(T)) return false;
    std::memcpy(&dst, src, sizeof(T));
    return true;
}
}  // namespace

cudaError_t ang_upload_tables(const void *tables, size_t size)
{
    ATab t;
    if (!unpack(t, tables, size)) return cudaErrorInvalidValue;
    return cudaMemcpyToSymbol(grpp_ang::grpp::c_tab, &t, sizeof(t));
}

cudaError_t ang_set_final_max_smem(int bytes)
{
    cudaError_t e = cudaFuncSetAttribute(grpp_ang::grpp::final_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(grpp_ang::grpp::final_kernel<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(grpp_ang::grpp::final_kernel<512>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    return e;
}

cudaError_t ang_final_occupancy(int nt, size_t smem, int *blocks_per_sm)
{
    if (nt == 128) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, grpp_ang::grpp::final_kernel<128>, 128, smem);
    if (nt == 256) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, grpp_ang::grpp::final_kernel<256>, 256, smem);
    if (nt == 512) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, grpp_ang::grpp::final_kernel<512>, 512, smem);
    return cudaErrorInvalidValue;
}

cudaError_t ang_launch_atab(int blocks, int threads, cudaStream_t s, int L, int l, double *out)
{
    grpp_ang::grpp::atab_kernel<<<blocks, threads, 0, s>>>(L, l, out);
    return cudaGetLastError();
}

cudaError_t ang_launch_oc_proj(int blocks, int threads, cudaStream_t s, const void *args, size_t size)
{
    AOcp a;
    if (!unpack(a, args, size)) return cudaErrorInvalidValue;
    grpp_ang::grpp::oc_proj_kernel<<<blocks, threads, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t ang_launch_omega_tab(int blocks, int threads, size_t smem, cudaStream_t s, const void *fin, size_t fin_size,
                                 const void *layout, size_t layout_size, const int *op_shell, const int *op_centre,
                                 int n_pairs, double *omtab)
{
    AFin f;
    ASmem m;
    if (!unpack(f, fin, fin_size) || !unpack(m, layout, layout_size) || threads != grpp_ang::grpp::kFinThreads)
        return cudaErrorInvalidValue;
    grpp_ang::grpp::omega_tab_kernel<<<blocks, threads, smem, s>>>(f, m, op_shell, op_centre, n_pairs, omtab);
    return cudaGetLastError();
}

cudaError_t nofma_launch_ftab(int blocks, int threads, size_t smem, cudaStream_t s, const void *rad, size_t rad_size,
                              double *ftab)
{
    ARad r;
    if (!unpack(r, rad, rad_size) || threads != grpp_ang::grpp::kRadThreads) return cudaErrorInvalidValue;
    grpp_ang::grpp::ftab_kernel<<<blocks, threads, smem, s>>>(r, ftab);
    return cudaGetLastError();
}

cudaError_t nofma_launch_wu_table(int blocks, int threads, cudaStream_t s, const void *rad, size_t rad_size, int n_grpps,
                                  double *wu)
{
    ARad r;
    if (!unpack(r, rad, rad_size)) return cudaErrorInvalidValue;
    grpp_ang::grpp::wu_table_kernel<<<blocks, threads, 0, s>>>(r, n_grpps, wu);
    return cudaGetLastError();
}

cudaError_t ang_launch_final(int nt, int blocks, size_t smem, cudaStream_t s, const void *fin, size_t fin_size,
                             const void *layout, size_t layout_size)
{
    AFin f;
    ASmem m;
    if (!unpack(f, fin, fin_size) || !unpack(m, layout, layout_size)) return cudaErrorInvalidValue;
    if (nt == 128) grpp_ang::grpp::final_kernel<128><<<blocks, 128, smem, s>>>(f, m);
    else if (nt == 256) grpp_ang::grpp::final_kernel<256><<<blocks, 256, smem, s>>>(f, m);
    else if (nt == 512) grpp_ang::grpp::final_kernel<512><<<blocks, 512, smem, s>>>(f, m);
    else return cudaErrorInvalidValue;
    return cudaGetLastError();
}

}  // namespace grpp
