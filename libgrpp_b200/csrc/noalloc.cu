// Allocation-free entry point: libgrpp_b200_type2_batch_noalloc.
//
// Some callers cannot let a library call cudaMalloc: applications whose device
// memory is owned by a pool or framework allocator (a cudaMalloc behind the
// allocator's back can fail once the pool holds the memory, and fragments what
// it does not), and long-running services that must keep the device footprint
// they had at start-up. This translation unit serves them: every device buffer
// it uses is file-scope static device memory, created when the library is
// loaded and held until the process exits:
//   * the constant tables the kernels read (Bessel, RSH, factorials, ...),
//   * one scratch array of kNoAllocScratchBytes (32 MiB) that holds a call's
//     packed inputs, the angular tensors, the radial tables and their per-entry
//     working state (running sums, screening estimates, flags), and the outputs
//     before they are copied back.
// The kernels are the engine's own radial and angular kernels, compiled here a
// second time (inside namespace grpp_noalloc) so that they read these static
// tables; no file of the regular path is changed.
//
// Behaviour:
//  * The batch is checked on the host before any CUDA call (indices, powers,
//    Cartesian lists); a malformed batch returns LIBGRPP_B200_ERR_INVALID.
//  * Set-up (tables copied with cudaMemcpyToSymbol, the scratch address taken
//    with cudaGetSymbolAddress) happens on the first call on each device, with
//    that device current; make that first call before any stream capture.
//  * The call is synchronous: it copies with cudaMemcpy and launches on the
//    legacy default stream, and returns when the results are on the host.
//  * A batch whose packed size exceeds the scratch array is rejected with
//    LIBGRPP_B200_ERR_INVALID and a message naming both sizes; nothing runs.
//  * All calls share the scratch array, which keeps the last call's contents.
//    Everything a call reads is written by that call first. Calls that overlap
//    on the GPU (from several host threads, or asynchronously) would race on
//    the array: host calls are serialised by a mutex, and each call returns
//    only after its results are on the host.
#include <cstdint>
#include <cstring>
#include <cmath>
#include <mutex>
#include <string>
#include <vector>
#include <algorithm>
#include <cuda_runtime.h>

#include "../../include/libgrpp.h"
#include "../../include/libgrpp_b200.h"
#include "tables.h"

namespace grpp_noalloc {
#include "grpp_common.cuh"
#include "specfunc.cuh"
#include "radial.cuh"
#include "angular.cuh"
}  // namespace grpp_noalloc

namespace grpp {
void set_error(int code, const std::string &msg);
}

namespace grpp_noalloc {
namespace {

using namespace grpp_noalloc::grpp;

constexpr size_t kNoAllocScratchBytes = 32u << 20;  // 32 MiB
constexpr int kMaxDevices = 64;

// static constant tables (sizes of tables.cpp's layout for kRshL = 32, kMaxL = 10)
constexpr size_t kNaBessel = (size_t)kBesNX * kBesL * 5;
constexpr size_t kNaRsh = 320705, kNaComb = 6545 * 3, kNaLmat = 6900;

static __device__ __align__(256) unsigned char g_scratch[kNoAllocScratchBytes];
static __device__ double g_bessel[kNaBessel];
static __device__ __align__(16) double g_bessel_p[kNaBessel];
static __device__ double g_rfun[kRfunL * kRfunL];
static __device__ double g_boys[kBoysNX * kBoysNN];
static __device__ double g_dawson[kDawNY];
static __device__ double g_rsh_coef[kNaRsh];
static __device__ int g_rsh_off[kRshL + 2];
static __device__ int8_t g_rsh_comb[kNaComb];
static __device__ int g_rsh_comb_off[kRshL + 2];
static __device__ double g_lmat[kNaLmat];
static __device__ int g_lmat_off[kMaxL + 3];
static __device__ double g_dfact[kDfMax + 2];
static __device__ double g_binom[kBinN * kBinN];

std::mutex g_mu;
bool g_ready[kMaxDevices] = {false};
unsigned char *g_scratch_ptr[kMaxDevices] = {nullptr};
::grpp::HostTables g_host;
bool g_host_ready = false;

#define NA_CUDA(call)                                                                                  \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess) {                                                                       \
            ::grpp::set_error(LIBGRPP_B200_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
            return LIBGRPP_B200_ERR_CUDA;                                                              \
        }                                                                                              \
    } while (0)

#define NA_CHECK(cond, msg)                                      \
    do {                                                         \
        if (!(cond)) {                                           \
            ::grpp::set_error(LIBGRPP_B200_ERR_INVALID, (msg));  \
            return LIBGRPP_B200_ERR_INVALID;                     \
        }                                                        \
    } while (0)

template <typename T, typename S>
int copy_table(const S &sym, const std::vector<T> &v, size_t cap, const T **dev)
{
    NA_CHECK(v.size() <= cap, "internal table larger than its static array");
    if (!v.empty()) NA_CUDA(cudaMemcpyToSymbol(sym, v.data(), v.size() * sizeof(T)));
    void *p = nullptr;
    NA_CUDA(cudaGetSymbolAddress(&p, sym));
    *dev = (const T *)p;
    return 0;
}

// once per device, with that device current
int setup(int dev)
{
    if (g_ready[dev]) return 0;
    if (!g_host_ready) {
        ::grpp::build_host_tables(g_host);
        g_host_ready = true;
    }
    const ::grpp::HostTables &h = g_host;
    DeviceTables d;
    d.grid = nullptr;  // grid points computed by the kernels themselves
    int rc = 0;
    if ((rc = copy_table(g_bessel, h.bessel, kNaBessel, &d.bessel))) return rc;
    if ((rc = copy_table(g_bessel_p, h.bessel_p, kNaBessel, &d.bessel_p))) return rc;
    if ((rc = copy_table(g_rfun, h.rfun, (size_t)kRfunL * kRfunL, &d.rfun))) return rc;
    if ((rc = copy_table(g_boys, h.boys, (size_t)kBoysNX * kBoysNN, &d.boys))) return rc;
    if ((rc = copy_table(g_dawson, h.dawson, (size_t)kDawNY, &d.dawson))) return rc;
    if ((rc = copy_table(g_rsh_coef, h.rsh_coef, kNaRsh, &d.rsh_coef))) return rc;
    if ((rc = copy_table(g_rsh_off, h.rsh_off, (size_t)kRshL + 2, &d.rsh_off))) return rc;
    if ((rc = copy_table(g_rsh_comb, h.rsh_comb, kNaComb, &d.rsh_comb))) return rc;
    if ((rc = copy_table(g_rsh_comb_off, h.rsh_comb_off, (size_t)kRshL + 2, &d.rsh_comb_off))) return rc;
    if ((rc = copy_table(g_lmat, h.lmat, kNaLmat, &d.lmat))) return rc;
    if ((rc = copy_table(g_lmat_off, h.lmat_off, (size_t)kMaxL + 3, &d.lmat_off))) return rc;
    if ((rc = copy_table(g_dfact, h.dfact, (size_t)kDfMax + 2, &d.dfact))) return rc;
    if ((rc = copy_table(g_binom, h.binom, (size_t)kBinN * kBinN, &d.binom))) return rc;
    NA_CUDA(cudaMemcpyToSymbol(c_tab, &d, sizeof(d)));
    void *p = nullptr;
    NA_CUDA(cudaGetSymbolAddress(&p, g_scratch));
    g_scratch_ptr[dev] = (unsigned char *)p;
    NA_CUDA(cudaFuncSetAttribute(radial_walk_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024));
    NA_CUDA(cudaFuncSetAttribute(final_kernel<kFinThreads>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    g_ready[dev] = true;
    return 0;
}

// bump layout of one call inside the scratch array
struct Arena {
    size_t used = 0;
    size_t take(size_t bytes)
    {
        const size_t o = (used + 255) & ~size_t(255);
        used = o + std::max<size_t>(bytes, 8);
        return o;
    }
};

double host_gaussian_norm(int L, double a) { return std::pow(2 * a / kPi, 0.75) * std::pow(4 * a, 0.5 * L); }

// Checks of every index and value the packing below reads, on the host and before any
// CUDA call: a malformed batch is rejected with LIBGRPP_B200_ERR_INVALID whether or not
// a device is present, and nothing is read outside the caller's arrays.
int validate(const libgrpp_b200_batch_t *b)
{
    NA_CHECK(b != nullptr && b->n_tasks >= 0, "null batch or negative task count");
    if (b->n_tasks == 0) return 0;
    NA_CHECK(b->n_shells > 0 && b->n_centres > 0 && b->n_grpps > 0 && b->n_pots >= 0, "empty batch description");
    for (int i = 0; i < b->n_shells; i++) {
        const int L = b->shell_L[i];
        NA_CHECK(L >= 0 && L <= kMaxL && b->shell_nprim[i] >= 1 && b->shell_nprim[i] <= kRadMaxPrims,
                 "shell outside the supported limits (L <= 10, 1..64 primitives)");
        NA_CHECK(b->shell_prim_off[i] >= 0 && b->shell_cart_off[i] >= 0, "negative shell offset");
        for (int q = 0; q < ncart(L); q++) {
            const int *c = b->cart_list + 3 * (b->shell_cart_off[i] + q);
            NA_CHECK(c[0] >= 0 && c[1] >= 0 && c[2] >= 0 && c[0] + c[1] + c[2] == L, "invalid Cartesian component list");
        }
    }
    for (int p = 0; p < b->n_pots; p++) {
        NA_CHECK(b->pot_L[p] >= 0 && b->pot_L[p] <= kMaxL, "potential angular momentum outside 0..10");
        NA_CHECK(b->pot_nprim[p] >= 0 && b->pot_prim_off[p] >= 0, "negative potential size or offset");
        for (int k = 0; k < b->pot_nprim[p]; k++) {
            const int n = b->pot_powers[b->pot_prim_off[p] + k];
            NA_CHECK(n >= 0 && n <= 2, "potential power n must be 0, 1 or 2");
        }
    }
    for (int g = 0; g < b->n_grpps; g++) {
        NA_CHECK(b->grpp_n_arep[g] >= 0 && b->grpp_arep_off[g] >= 0, "negative potential count or offset in a GRPP");
        for (int i = 0; i < b->grpp_n_arep[g]; i++) {
            const int pot = b->grpp_pot_list[b->grpp_arep_off[g] + i];
            NA_CHECK(pot >= 0 && pot < b->n_pots, "GRPP potential index out of range");
        }
    }
    for (int c = 0; c < b->n_centres; c++)
        NA_CHECK(b->centre_grpp[c] >= 0 && b->centre_grpp[c] < b->n_grpps, "centre GRPP index out of range");
    for (int64_t t = 0; t < b->n_tasks; t++)
        NA_CHECK(b->task_a[t] >= 0 && b->task_a[t] < b->n_shells && b->task_b[t] >= 0 && b->task_b[t] < b->n_shells &&
                     b->task_c[t] >= 0 && b->task_c[t] < b->n_centres,
                 "task index out of range");
    return 0;
}

int run(const libgrpp_b200_batch_t *b, double *h_arep)
{
    if (int rc = validate(b)) return rc;
    if (b->n_tasks == 0) return 0;
    int dev = 0;
    NA_CUDA(cudaGetDevice(&dev));
    NA_CHECK(dev >= 0 && dev < kMaxDevices, "device index out of range");
    std::lock_guard<std::mutex> lk(g_mu);
    int rc = setup(dev);
    if (rc) return rc;
    const int64_t nt = b->n_tasks;
    const int ns = b->n_shells;

    // ---- shells, radial primitives (shrunk and normalised), Cartesian lists
    std::vector<int> sh_L(b->shell_L, b->shell_L + ns), sh_np(b->shell_nprim, b->shell_nprim + ns),
        sh_po(b->shell_prim_off, b->shell_prim_off + ns), sh_co(ns), rp_off(ns), rp_n(ns);
    std::vector<double> sh_or(b->shell_origin, b->shell_origin + 3 * ns), rp_c, rp_a, pc, pa;
    std::vector<int8_t> cart;
    int total_prims = 0;
    for (int i = 0; i < ns; i++) {
        NA_CHECK(sh_L[i] >= 0 && sh_L[i] <= kMaxL && sh_np[i] >= 1 && sh_np[i] <= kRadMaxPrims,
                 "shell outside the supported limits (L <= 10, 1..64 primitives)");
        total_prims = std::max(total_prims, sh_po[i] + sh_np[i]);
    }
    pc.assign(b->prim_coef, b->prim_coef + total_prims);
    pa.assign(b->prim_alpha, b->prim_alpha + total_prims);
    for (int i = 0; i < ns; i++) {
        sh_co[i] = (int)(cart.size() / 3);
        for (int q = 0; q < 3 * ncart(sh_L[i]); q++) cart.push_back((int8_t)b->cart_list[3 * b->shell_cart_off[i] + q]);
        rp_off[i] = (int)rp_c.size();
        for (int k = 0; k < sh_np[i]; k++) {
            const double c = pc[sh_po[i] + k], a = pa[sh_po[i] + k];
            if (std::fabs(c) > kZeroThresh) {
                rp_c.push_back(c * host_gaussian_norm(sh_L[i], a));
                rp_a.push_back(a);
            }
        }
        rp_n[i] = (int)rp_c.size() - rp_off[i];
    }
    // ---- potentials (|c| < 1e-14 dropped) and the AREP lists of every GRPP
    const int np = b->n_pots;
    std::vector<int> p_L(np), p_n(np), p_off(np), p_pw, g_sl_off(b->n_grpps), g_sl_n(b->n_grpps), g_zero(b->n_grpps, 0), sl_pot;
    std::vector<double> p_c, p_a;
    for (int p = 0; p < np; p++) {
        p_L[p] = b->pot_L[p];
        p_off[p] = (int)p_c.size();
        for (int k = 0; k < b->pot_nprim[p]; k++) {
            const int o = b->pot_prim_off[p] + k;
            if (std::fabs(b->pot_coef[o]) < kZeroThresh) continue;
            p_pw.push_back(b->pot_powers[o]);
            p_c.push_back(b->pot_coef[o]);
            p_a.push_back(b->pot_alpha[o]);
        }
        p_n[p] = (int)p_c.size() - p_off[p];
    }
    for (int g = 0; g < b->n_grpps; g++) {
        g_sl_off[g] = (int)sl_pot.size();
        g_sl_n[g] = b->grpp_n_arep[g];
        NA_CHECK(g_sl_n[g] <= kRadMaxPots, "more than 24 averaged potentials in one GRPP");
        int nterm = 0;
        for (int i = 0; i < g_sl_n[g]; i++) {
            const int pot = b->grpp_pot_list[b->grpp_arep_off[g] + i];
            NA_CHECK(p_L[pot] >= 0 && p_L[pot] <= kMaxL, "potential angular momentum outside 0..10");
            sl_pot.push_back(pot);
            nterm += p_n[pot];
        }
        NA_CHECK(nterm <= kRadMaxTerms, "more than 256 averaged potential terms in one GRPP");
    }
    // ---- tasks, radial items, angular tensors needed
    std::vector<int> ta(b->task_a, b->task_a + nt), tb(b->task_b, b->task_b + nt), tc(b->task_c, b->task_c + nt), rad_task;
    std::vector<int64_t> out_off(nt + 1, 0), q_off(nt, -1), rad_q;
    std::vector<uint8_t> has_ul(nt, 0);
    std::vector<int> no_proj(nt, -1);
    std::vector<std::pair<int, int>> atab_need;
    int64_t qtot = 0;
    int l1m = 0, l2m = 0, dn = 1, npot = 0, fin_lam = 0, fin_nq = 1;
    for (int64_t t = 0; t < nt; t++) {
        NA_CHECK(ta[t] >= 0 && ta[t] < ns && tb[t] >= 0 && tb[t] < ns && tc[t] >= 0 && tc[t] < b->n_centres, "task index out of range");
        const int la = sh_L[ta[t]], lb = sh_L[tb[t]], g = b->centre_grpp[tc[t]];
        NA_CHECK(ncart(la) * ncart(lb) <= kFinThreads * kFinElemPerThread, "shell pair block larger than 1024 Cartesian pairs");
        out_off[t + 1] = out_off[t] + (int64_t)ncart(la) * ncart(lb);
        if (g_sl_n[g] == 0) continue;
        int64_t e = 0;
        for (int i = 0; i < g_sl_n[g]; i++) {
            const int L = p_L[sl_pot[g_sl_off[g] + i]];
            e += (int64_t)(L + la + 1) * (L + lb + 1) * (la + lb + 1);
            l1m = std::max(l1m, L + la);
            l2m = std::max(l2m, L + lb);
            fin_lam = std::max(fin_lam, L + std::max(la, lb));
            fin_nq = std::max(fin_nq, (L + la + 1) * (L + lb + 1) * (la + lb + 1));
            atab_need.push_back({L, la});
            atab_need.push_back({L, lb});
        }
        NA_CHECK(e <= kRadMaxEntries, "radial table larger than 16384 entries for one task");
        q_off[t] = qtot;
        rad_task.push_back((int)t);
        rad_q.push_back(qtot);
        qtot += e;
        dn = std::max(dn, la + lb + 1);
        npot = std::max(npot, g_sl_n[g]);
    }
    NA_CHECK(std::max(l1m, l2m) <= kRadMaxLam && dn <= kRadMaxN, "angular momentum too high for the radial path");
    std::sort(atab_need.begin(), atab_need.end());
    atab_need.erase(std::unique(atab_need.begin(), atab_need.end()), atab_need.end());
    std::vector<int64_t> atab_off((kMaxL + 2) * (kMaxL + 2), -1);
    int64_t atab_tot = 0;
    for (auto &lp : atab_need) {
        atab_off[lp.first * (kMaxL + 2) + lp.second] = atab_tot;
        atab_tot += atab_size(lp.first, lp.second);
    }
    const int64_t out_tot = out_off[nt];

    // ---- layout inside the scratch array
    std::vector<double> c_or(b->centre_origin, b->centre_origin + 3 * b->n_centres);
    std::vector<int> c_g(b->centre_grpp, b->centre_grpp + b->n_centres), n_arep_v(b->n_grpps);
    for (int g = 0; g < b->n_grpps; g++) n_arep_v[g] = g_sl_n[g];
    std::vector<char> host;
    Arena ar;
    auto put = [&](const void *src, size_t bytes) {
        const size_t o = ar.take(bytes);
        if (host.size() < ar.used) host.resize(ar.used);
        if (bytes) memcpy(host.data() + o, src, bytes);
        return o;
    };
#define PUT(v) put((v).data(), (v).size() * sizeof((v)[0]))
    const size_t o_shL = PUT(sh_L), o_shnp = PUT(sh_np), o_shpo = PUT(sh_po), o_shco = PUT(sh_co), o_pa = PUT(pa),
                 o_pc = PUT(pc), o_sor = PUT(sh_or), o_cart = PUT(cart), o_rpo = PUT(rp_off), o_rpn = PUT(rp_n),
                 o_rpc = PUT(rp_c), o_rpa = PUT(rp_a), o_pL = PUT(p_L), o_pn = PUT(p_n), o_poff = PUT(p_off),
                 o_ppw = PUT(p_pw), o_pcoef = PUT(p_c), o_palpha = PUT(p_a), o_gslo = PUT(g_sl_off), o_gsln = PUT(g_sl_n),
                 o_gnar = PUT(n_arep_v), o_slp = PUT(sl_pot), o_gz = PUT(g_zero), o_cor = PUT(c_or), o_cg = PUT(c_g),
                 o_ta = PUT(ta), o_tb = PUT(tb), o_tc = PUT(tc), o_too = PUT(out_off), o_thul = PUT(has_ul),
                 o_tqo = PUT(q_off), o_np = PUT(no_proj), o_rt = PUT(rad_task), o_rq = PUT(rad_q), o_aoff = PUT(atab_off);
#undef PUT
    const size_t in_bytes = ar.used;
    const int64_t qn = std::max<int64_t>(qtot, 1);
    const size_t o_atab = ar.take(atab_tot * sizeof(double)), o_Q = ar.take(qn * sizeof(double)),
                 o_Sp = ar.take(qn * sizeof(double)), o_scr = ar.take(qn * sizeof(double)), o_ef = ar.take(qn),
                 o_walk = ar.take(rad_task.size() + 1), o_arep = ar.take(out_tot * sizeof(double)),
                 o_dummy = ar.take(out_tot * sizeof(double));
    if (ar.used > kNoAllocScratchBytes) {
        ::grpp::set_error(LIBGRPP_B200_ERR_INVALID,
                          "batch needs " + std::to_string(ar.used) + " bytes of device memory; the allocation-free entry point has " +
                              std::to_string(kNoAllocScratchBytes) + " (split the batch)");
        return LIBGRPP_B200_ERR_INVALID;
    }
    unsigned char *base = g_scratch_ptr[dev];
    NA_CUDA(cudaMemcpy(base, host.data(), in_bytes, cudaMemcpyHostToDevice));
    auto P = [&](size_t o) { return (void *)(base + o); };

    int nsm = 0;
    NA_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    for (auto &lp : atab_need) {
        const int64_t sz = atab_size(lp.first, lp.second);
        const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((sz + 255) / 256, 4096));
        atab_kernel<<<blocks, 256>>>(lp.first, lp.second,
                                     (double *)P(o_atab) + atab_off[lp.first * (kMaxL + 2) + lp.second]);
        NA_CUDA(cudaGetLastError());
    }
    if (!rad_task.empty()) {
        RadialArgs r{};
        memset(&r, 0, sizeof(r));
        r.n_items = (int)rad_task.size();
        r.item_task = (const int *)P(o_rt);
        r.task_a = (const int *)P(o_ta);
        r.task_b = (const int *)P(o_tb);
        r.task_c = (const int *)P(o_tc);
        r.shell_L = (const int *)P(o_shL);
        r.shell_origin = (const double *)P(o_sor);
        r.rp_off = (const int *)P(o_rpo);
        r.rp_n = (const int *)P(o_rpn);
        r.rp_coef = (const double *)P(o_rpc);
        r.rp_alpha = (const double *)P(o_rpa);
        r.shell_nprim = (const int *)P(o_shnp);
        r.shell_prim_off = (const int *)P(o_shpo);
        r.prim_coef = (const double *)P(o_pc);
        r.prim_alpha = (const double *)P(o_pa);
        r.centre_origin = (const double *)P(o_cor);
        r.centre_grpp = (const int *)P(o_cg);
        r.grpp_sl_off = (const int *)P(o_gslo);
        r.grpp_sl_n = (const int *)P(o_gsln);
        r.sl_pot = (const int *)P(o_slp);
        r.pot_L = (const int *)P(o_pL);
        r.pot_nprim = (const int *)P(o_pn);
        r.pot_prim_off = (const int *)P(o_poff);
        r.pot_powers = (const int *)P(o_ppw);
        r.pot_coef = (const double *)P(o_pcoef);
        r.pot_alpha = (const double *)P(o_palpha);
        r.q_off = (const int64_t *)P(o_rq);
        r.Q = (double *)P(o_Q);
        r.S_prev = (double *)P(o_Sp);
        r.scr = (double *)P(o_scr);
        r.eflag = (uint8_t *)P(o_ef);
        r.walk = (uint8_t *)P(o_walk);
        radial_screen_kernel<<<(int)std::min<int64_t>((int64_t)rad_task.size(), (int64_t)nsm * 32), kRadThreads>>>(r);
        NA_CUDA(cudaGetLastError());
        const size_t smem = (size_t)(npot + (l1m + 1) + (l2m + 1) + dn) * kRadRow * sizeof(double);
        radial_walk_kernel<<<(int)std::min<int64_t>((int64_t)rad_task.size(), (int64_t)nsm * 16), kRadThreads, smem>>>(r);
        NA_CUDA(cudaGetLastError());
    }
    FinalArgs f{};
    memset(&f, 0, sizeof(f));
    f.n_tasks = (int)nt;
    f.task_a = (const int *)P(o_ta);
    f.task_b = (const int *)P(o_tb);
    f.task_c = (const int *)P(o_tc);
    f.task_out_off = (const int64_t *)P(o_too);
    f.task_has_ul = (const uint8_t *)P(o_thul);
    f.task_q_off = (const int64_t *)P(o_tqo);
    f.task_proj_a = (const int *)P(o_np);
    f.task_proj_b = (const int *)P(o_np);
    f.shell_L = (const int *)P(o_shL);
    f.shell_cart_off = (const int *)P(o_shco);
    f.shell_prim_off = (const int *)P(o_shpo);
    f.prim_alpha = (const double *)P(o_pa);
    f.shell_origin = (const double *)P(o_sor);
    f.cart = (const int8_t *)P(o_cart);
    f.centre_origin = (const double *)P(o_cor);
    f.centre_grpp = (const int *)P(o_cg);
    f.grpp_sl_off = (const int *)P(o_gslo);
    f.grpp_sl_n = (const int *)P(o_gsln);
    f.grpp_n_arep = (const int *)P(o_gnar);
    f.sl_pot = (const int *)P(o_slp);
    f.grpp_oc_off = (const int *)P(o_gz);
    f.grpp_n_oc = (const int *)P(o_gz);
    f.pot_L = (const int *)P(o_pL);
    f.Q = (const double *)P(o_Q);
    f.atab_off = (const int64_t *)P(o_aoff);
    f.atab = (const double *)P(o_atab);
    f.arep = (double *)P(o_arep);
    f.so_x = f.so_y = f.so_z = (double *)P(o_dummy);  // no spin-orbit potentials: written with zeros
    FinalSmem fs{};
    fs.rsh_stride = 2 * fin_lam + 1;
    fs.n_rsh = (fin_lam + 1) * fs.rsh_stride;
    int n_om = 1, nabmax = 1;
    for (auto &lp : atab_need) {
        n_om = std::max(n_om, n_abc(lp.second) * lam_slots(lp.first, lp.second) * (2 * lp.first + 1));
        nabmax = std::max(nabmax, n_abc(lp.second));
    }
    fs.n_omega = n_om;
    fs.n_q = fin_nq;
    fs.n_v = std::max(6144, 3 * nabmax);
    const size_t smem = (size_t)(2 * fs.n_rsh + 2 * fs.n_omega + fs.n_q + fs.n_v) * sizeof(double);
    final_kernel<kFinThreads><<<(int)std::min<int64_t>(nt, (int64_t)nsm * 8), kFinThreads, smem>>>(f, fs);
    NA_CUDA(cudaGetLastError());
    NA_CUDA(cudaMemcpy(h_arep, P(o_arep), out_tot * sizeof(double), cudaMemcpyDeviceToHost));
    return 0;
}

}  // namespace
}  // namespace grpp_noalloc

#pragma GCC visibility push(default)
extern "C" int libgrpp_b200_type2_batch_noalloc(const libgrpp_b200_batch_t *batch, double *arep)
{
    ::grpp::set_error(0, "");
    if (!libgrpp_is_initialized()) {
        ::grpp::set_error(LIBGRPP_B200_ERR_NOT_INIT, "libgrpp_init() was not called");
        return LIBGRPP_B200_ERR_NOT_INIT;
    }
    return grpp_noalloc::run(batch, arep);
}
#pragma GCC visibility pop
